"""CPU checks of the drivers' file formats (names, CSV header, log lines)."""
from qed2d import drivers


def test_checkpoint_name_matches_reference_pattern():
    # configs/config_$(L1)_$(L2)_b$(beta)_m$(am0)_n$(i)  (main/hmc-nf2.jl:142-145)
    p = drivers._config_name("runs/", 64, 32, 4.0, 0.1, 200)
    assert p.endswith("configs/config_64_32_b4.0_m0.1_n200")


def test_hmc_log_line_format():
    class I:
        accepted, hini, hfin, dH = 1, 100.5, 100.25, -0.25
    line = drivers._hmc_line(I(), [1, 0, 1, 1])
    assert line == "    ACCEPT: Energy [inital: 100.5; final: 100.25; difference: -0.25]; Pacc = 0.75"
