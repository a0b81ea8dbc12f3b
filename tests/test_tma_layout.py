"""CPU checks of the TMA-staged batched solver's copy geometry (batch schedule 7).

The kernel (dav-qed2d_b200/csrc/batch_cg_uniform.cuh: UStage, tma_issue) loads,
for each tile of 32 x TY sites of replica r, five boxes of each staged spinor
field and four link boxes.  A TMA copy must start at an x coordinate whose byte
offset is a multiple of 16 and here must also lie inside the tensor (no copy
relies on out-of-bounds fill).  This restates the coordinate arithmetic and
checks, for every tile of the lattices the schedule accepts (L1 % 32 == 0,
L2 % TY == 0), alignment, bounds and that each halo box holds the periodic
neighbour the stencil reads; plus the stage layout: 128-byte aligned
destinations and transaction byte counts equal to the boxes' bytes.
"""
import pytest

F4, F2 = 16, 8          # bytes of a float4 spinor site and of a float2 link
FLOAT = 4               # the tensor maps' element: float32


def stage(ty):
    C, K, W = ty * 32 * F4, ty * F4, 32 * F4
    field = C + 2 * K + 2 * W
    u1c = 2 * field
    u1l = u1c + ty * 32 * F2
    u2c = u1l + ty * 16
    u2b = u2c + ty * 32 * F2
    total = u2b + 32 * F2
    return dict(C=C, K=K, W=W, FIELD=field, U1C=u1c, U1L=u1l, U2C=u2c, U2B=u2b, BYTES=total, LINKS=total - u1c)


def boxes(B, L1, L2, ty, r, t1, t2, nf):
    """(name, x, y, bx, by, nx, ny) of every copy tma_issue makes, in float32 units."""
    ny = B * L2
    y = r * L2 + t2 * ty
    ylo = r * L2 + (L2 - 1 if t2 == 0 else t2 * ty - 1)
    yhi = r * L2 + (0 if (t2 + 1) * ty == L2 else (t2 + 1) * ty)
    xl = L1 - 1 if t1 == 0 else 32 * t1 - 1
    xr = (32 * t1 + 32) % L1
    out = []
    for _ in range(nf):
        out += [("fc", 128 * t1, y, 128, ty, 4 * L1, ny), ("fk_left", 4 * xl, y, 4, ty, 4 * L1, ny),
                ("fk_right", 4 * xr, y, 4, ty, 4 * L1, ny), ("fw_low", 128 * t1, ylo, 128, 1, 4 * L1, ny),
                ("fw_high", 128 * t1, yhi, 128, 1, 4 * L1, ny)]
    out += [("u1c", 64 * t1, y, 64, ty, 2 * L1, ny),
            ("u1l", 2 * (L1 - 2 if t1 == 0 else 32 * t1 - 2), y, 4, ty, 2 * L1, ny),
            ("u2c", 64 * t1, y, 64, ty, 2 * L1, ny), ("u2b", 64 * t1, ylo, 64, 1, 2 * L1, ny)]
    return out


SHAPES = [(4, 512, 512), (2, 64, 48), (3, 64, 48), (2, 96, 40), (1, 32, 16), (5, 256, 128), (8, 128, 64)]


@pytest.mark.parametrize("ty", [8, 16])
@pytest.mark.parametrize("B,L1,L2", SHAPES)
def test_tma_boxes_aligned_inside_and_periodic(B, L1, L2, ty):
    if L1 % 32 or L2 % ty:
        pytest.skip("schedule 7 is not offered for this lattice at this tile height")
    s = stage(ty)
    for r in range(B):
        for t2 in range(L2 // ty):
            for t1 in range(L1 // 32):
                for nf in (1, 2):
                    got = 0
                    for name, x, y, bx, by, nx, ny in boxes(B, L1, L2, ty, r, t1, t2, nf):
                        assert (x * FLOAT) % 16 == 0, (name, x)
                        assert (bx * FLOAT) % 16 == 0 and bx <= 256 and by <= 256
                        assert 0 <= x and x + bx <= nx, (name, x, bx, nx)
                        assert r * L2 <= y and y + by <= (r + 1) * L2 <= ny, (name, y, by)
                        got += bx * by * FLOAT
                    assert got == nf * s["FIELD"] + s["LINKS"]
                # halos are the periodic neighbours inside replica r
                i1, i2 = 32 * t1, t2 * ty
                bx = dict((b[0], b) for b in boxes(B, L1, L2, ty, r, t1, t2, 1))
                assert bx["fk_left"][1] // 4 == (i1 - 1) % L1
                assert bx["fk_right"][1] // 4 == (i1 + 32) % L1
                assert bx["fw_low"][2] - r * L2 == (i2 - 1) % L2
                assert bx["fw_high"][2] - r * L2 == (i2 + ty) % L2
                first = bx["u1l"][1] // 2   # the box holds sites first, first + 1 of the row
                assert first + 1 < L1 and first + 1 == (i1 - 1) % L1
                assert bx["u2b"][2] - r * L2 == (i2 - 1) % L2


@pytest.mark.parametrize("ty", [8, 16])
def test_tma_stage_layout(ty):
    s = stage(ty)
    for key in ("C", "K", "W", "FIELD", "U1C", "U1L", "U2C", "U2B"):
        assert s[key] % 128 == 0, key
    # two stages and the alignment slack fit two 512-thread blocks per SM (228 KB)
    assert 2 * (2 * s["BYTES"] + 128 + 6456) <= 228 * 1024
