"""The four drivers end to end on small lattices: outputs in the reference's
formats, checkpoint written and resumed (main/hmc-nf2.jl:93-145)."""
import json
import os

import numpy as np
import pytest

from bdio_reader import read_bdio

pytestmark = pytest.mark.gpu


def write(path, d):
    with open(path, "w") as fh:
        json.dump(d, fh)
    return str(path)


def test_hmc_nf2_driver_checkpoint_and_resume(tmp_path):
    from qed2d import drivers
    inp = write(tmp_path / "nf2.in", {"Run": {"user": "u", "host": "h", "name": "t", "seed": 42},
                                       "Lattice": {"size": [8, 8], "beta": 4.0},
                                       "HMC": {"tau": 0.5, "ns": 4, "nthm": 0, "ntraj": 100, "Qzero": False,
                                               "mass": 0.5}})
    sd = str(tmp_path) + "/"
    drivers.main(["hmc-nf2", "-i", inp, "--savedir", sd, "--cont", "0"])
    rows = open(sd + "statistics.txt").read().splitlines()
    assert rows[0] == "step,accepted,plaquette,top_charge,acc_rate" and len(rows) == 101
    ck = sd + "configs/config_8_8_b4.0_m0.5_n100"
    assert os.path.exists(ck) and len(open(ck).read().splitlines()) == 128
    inp2 = write(tmp_path / "nf2b.in", {"Run": {"user": "u", "host": "h", "name": "t", "seed": 43},
                                         "Lattice": {"size": [8, 8], "beta": 4.0},
                                         "HMC": {"tau": 0.5, "ns": 4, "nthm": 0, "ntraj": 2, "Qzero": False,
                                                 "mass": 0.5}})
    drivers.main(["hmc-nf2", "-i", inp2, "--savedir", sd, "--cont", "100"])
    rows = open(sd + "statistics.txt").read().splitlines()
    assert [r.split(",")[0] for r in rows[-2:]] == ["101", "102"]
    assert "Continue HMC run from n=100" in open(sd + "log.txt").read()


def test_mc_rhmc_master_field_drivers(tmp_path, monkeypatch):
    from qed2d import drivers
    monkeypatch.chdir(tmp_path)
    mc = write(tmp_path / "mc.in", {"Run": {"user": "u", "host": "h", "name": "mc", "seed": 1234},
                                     "Lattice": {"size": [16, 16], "beta": 4.0},
                                     "HMC": {"ns": 5, "eps": 0.1, "nthm": 2, "ntraj": 3, "Qzero": False}})
    drivers.main(["mc", "-i", mc])
    assert "MEASUREMENT Trajectory 3 / 3" in open("mc.log").read()
    h, recs = read_bdio("mc.bdio")
    data = [r for r in recs if r["uinfo"] != 7]
    assert [r["uinfo"] for r in data] == [1, 2, 3, 4]
    assert np.array_equal(np.frombuffer(data[1]["data"], "<f8"), [16, 16, 4.0, 3])
    pl = np.frombuffer(data[2]["data"], "<f8").reshape(16, 3)   # the series, written L1 times
    qt = np.frombuffer(data[3]["data"], "<f8").reshape(16, 3)
    assert (pl == pl[0]).all() and (qt == qt[0]).all() and (0 < pl).all() and (pl < 1).all()
    assert np.abs(qt - np.rint(qt)).max() < 1e-9
    rh = write(tmp_path / "rh.in", {"Run": {"user": "u", "host": "h", "name": "rh", "seed": 7},
                                     "Lattice": {"size": [8, 8], "beta": 5.0},
                                     "HMC": {"tau": 0.5, "ns": 4, "nthm": 0, "ntraj": 2, "Qzero": False},
                                     "RHMC": {"masses": [0.5], "n_rhmc": [3], "r_a_g5Dw_sqr": [0.05],
                                              "r_b_g5Dw_sqr": [30.0]}})
    sd = str(tmp_path / "rh") + "/"
    drivers.main(["rhmc", "-i", rh, "--savedir", sd, "--power-iter", "50"])
    rows = open(sd + "statistics.txt").read().splitlines()
    assert rows[0] == "step,accepted,plaquette,top_charge,reweight_factor,lambda_min,lambda_max,acc_rate"
    assert len(rows) == 3 and all(len(r.split(",")) == 8 for r in rows)
    mf = write(tmp_path / "mf.in", {"Run": {"user": "u", "host": "h", "name": "mf", "seed": 1234,
                                             "measurements": 1},
                                     "Lattice": {"size": [64, 64], "beta": 11.25},
                                     "HMC": {"ns": 5, "eps": 0.05, "ntraj": 1, "Qzero": False}})
    drivers.main(["master-field", "-i", mf])
    h, recs = read_bdio("mf.bdio")
    data = [r for r in recs if r["uinfo"] != 7]
    assert [r["uinfo"] for r in data] == [1, 2, 3, 4, 3, 4]   # two measurements (before and after)
    assert np.array_equal(np.frombuffer(data[1]["data"], "<f8"), [64, 64, 11.25, 1])
    for j in (0, 1):
        p = np.frombuffer(data[2 + 2 * j]["data"], "<f8")
        q = np.frombuffer(data[3 + 2 * j]["data"], "<f8")
        assert p.size == 64 * 64 and q.size == 64 * 64
        assert (np.abs(p) <= 1).all() and (np.abs(q) <= np.pi).all()
        Q = q.sum() / (2 * np.pi)
        assert abs(Q - round(Q)) < 1e-9
    assert "Plaquette and error:" in open("mf.log").read()
