"""The bench's roofline denominators (no GPU): the path-grouped algorithmic bytes per depth map,
B_alg = (S+1) N + 3 e V + 8 V + 60 N, reproduce the published table for every configuration
(FP32 and FP16 volumes), the cost kernel's algorithmic work is 144 flop per voxel and source,
and the SGM stage's byte model counts what the pair kernels and the combine must move."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402

# (W, H, D, S) -> (B_alg FP32, B_alg FP16) in MB, as published for this metric
TABLE = {(320, 240, 64, 4): (103.3, 73.8), (640, 480, 128, 5): (806.7, 570.8),
         (752, 480, 128, 5): (947.9, 670.7), (1280, 720, 192, 4): (3599.0, 2537.0)}


@pytest.fixture
def shape(monkeypatch):
    def set_shape(W, H, D, S):
        for k, v in dict(W=W, H=H, D=D, S=S).items():
            monkeypatch.setattr(bench, k, v)
    return set_shape


@pytest.mark.parametrize("cfg", list(TABLE))
def test_b_alg_matches_the_published_table(shape, cfg):
    shape(*cfg)
    for e, want in ((4, TABLE[cfg][0]), (2, TABLE[cfg][1])):
        b_alg, _ = bench.algorithmic_bytes(e)
        assert abs(b_alg / 1e6 - want) <= 0.05 * (1 if want < 1000 else 10), (cfg, e, b_alg)


def test_cost_and_sgm_work_at_the_headline_shape(shape):
    shape(640, 480, 128, 5)
    N, V = 640 * 480, 640 * 480 * 128
    flop, tex_flop, nbytes = bench.cost_kernel_work(4)
    assert flop == 144 * V * 5 == 28_311_552_000 and tex_flop == 0
    assert nbytes == 4 * V + 4 * N + 16 * N * 5            # volume once, reference, 5 quad images
    simt, tex, nb16 = bench.cost_kernel_work(2, texels=True)
    assert nb16 == 2 * V + 4 * N + 4 * N * 5
    # the texture unit takes the nine bilinear interpolations (6 flop each) off the SIMT pipes
    assert tex == 54 * V * 5 and simt + tex == 144 * V * 5
    # the SGM + winner-take-all + fusion share of B_alg: two sweeps over C, the forward sum
    # written and read once, the reference image, fusion state and outputs
    assert bench.sgm_alg_bytes(4) == 16 * V + 60 * N and bench.sgm_alg_bytes(2) == 12 * V + 60 * N
    _, sgm16 = bench.algorithmic_bytes(2)   # the FP16 form's pair volumes are FP16 as well
    assert abs(sgm16 / V - 48) < 0.5
    _, sgm = bench.algorithmic_bytes(4)
    # 8 paths read C and the reference; 4 pair volumes stored, reduced into (read + write) and
    # read once by the combine; depth and index written
    assert sgm == 8 * (4 * V + 4 * N) + 4 * (4 * V + 8 * V) + 4 * 4 * V + 8 * N
    assert abs(sgm / V - 96) < 0.5                        # ~96 bytes per voxel for FP32


def test_texture_fetch_model(shape):
    """Fetches of one cost launch with a texture sampler: the tile design issues 52 fetch
    instructions per warp and source in reference mode (10 row samples + 16 corrupted-neighbour
    samples per plane pair), 20 with corrected samples; the algorithmic count is 3 (1) per voxel
    and source.  At 640x480x128x5 that is 21,964,800 warp fetch instructions, the figure the ncu
    capture of the FP16 texture kernel shows as 8 texture requests each (172.6 M requests; the
    partly idle last tile column issues a little less)."""
    shape(640, 480, 128, 5)
    V = 640 * 480 * 128
    alg, issued = bench.cost_kernel_fetches(True)
    assert alg == 3 * V * 5 and issued == 22 * 60 * 8 * 8 * 5 * 52 * 32 == 21_964_800 * 32
    alg1, issued1 = bench.cost_kernel_fetches(False)
    assert alg1 == V * 5 and issued1 * 52 == issued * 20
    assert 8 * issued / 32 >= 172_646_400   # no more requests than instructions allow


def test_cost_roofline_binding_roof(shape):
    """The bench line's `roofline`: the texture unit for a texture sampler (algorithmic fetches over
    the kernel time against 148 x 4 fetches per clock), the FP32 SIMT pipes for exact bilinear."""
    shape(640, 480, 128, 5)
    r = bench.cost_roofline(0.6865, 0.7185, 2, True, True, 1965.0, 6441.6, "measured", "fp16", 55183104)
    assert r["bound"] == "texture" and r["unit"] == "G fetches/s" and r["traffic"] == 55183104
    assert abs(r["peak"] - 148 * 4 * 1.965) < 1e-6
    assert abs(r["frac"] - 589_824_000 / 0.6865e-3 / 1e9 / r["peak"]) < 1e-9 and 0.73 < r["frac"] < 0.74
    assert 0.87 < r["frac_issued"] < 0.89
    f = r["fp32_simt"]
    assert f["bound"] == "fp32" and abs(f["frac"] - 17_694_720_000 / 0.6865e-3 / 1e12 / f["peak"]) < 1e-9
    r32 = bench.cost_roofline(1.112, 1.114, 4, False, True, 1965.0, 6441.6, "measured", "fp32", 161212928)
    assert r32["bound"] == "fp32" and "fp32_simt" not in r32 and 0.34 < r32["frac"] < 0.35
    assert r32["ms_per_launch"] == 1.112 and r32["traffic"] == 161212928
    assert bench.cost_roofline(0.0, 0.0, 2, True, True, 1965.0, 6441.6, "measured", "fp16", None)["frac"] is None
