"""Device-resident sketch object: top-K recovery without the dense estimate
equals the dense path's top-K exactly (same entries, values and order),
for one tile and for many small tiles; listed-entry queries equal the dense
estimate bit for bit; and both against the CPU oracle."""
import numpy as np
import pytest

from compmatmul_b200 import device
from compmatmul_b200.planted import planted_problem
from compmatmul_b200.sketch import Sketch


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["fft", "fwht"])
def test_sketch_topk_equals_dense_topk(gpu, variant):
    import torch
    AT, B, (pi, pk, pj) = planted_problem(700, 500, 900, 40, 1234)
    dAT, dB = torch.from_numpy(AT).cuda(), torch.from_numpy(B).cuda()
    s = Sketch.compute(dAT, dB, 7, 4096, 99, variant)
    C = s.dense()
    di, dj, dv = device.topk(C, 40)
    for scratch in (0, 64 * 1024):  # one tile; tiles of ~9 rows
        ti, tj, tv = s.topk(40, scratch_bytes=scratch)
        np.testing.assert_array_equal(ti, di)
        np.testing.assert_array_equal(tj, dj)
        np.testing.assert_array_equal(tv, dv)
    assert set(zip(ti.tolist(), tj.tolist())) == set(zip(pi.tolist(), pj.tolist()))
    rng = np.random.default_rng(5)
    qi, qj = rng.integers(0, 700, 500), rng.integers(0, 900, 500)
    np.testing.assert_array_equal(s.entries(qi, qj), C.cpu().numpy()[qi, qj])


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["fft", "fwht"])
def test_sketch_estimates_match_oracle(gpu, oracle, variant):
    """The device sketch object's listed-entry queries and top-K against the
    CPU oracle's sketch and median estimates on the same inputs."""
    import torch
    AT, B, _ = planted_problem(300, 200, 260, 16, 4321)
    s = Sketch.compute(torch.from_numpy(AT).cuda(), torch.from_numpy(B).cuda(), 5, 4096, 31, variant)
    p = oracle.compressed_product(variant, None, AT, B, 5, 4096, 31)
    want = oracle.decompress(variant, None, p, 5, 4096, 31, 300, 260)
    rng = np.random.default_rng(9)
    qi, qj = rng.integers(0, 300, 400), rng.integers(0, 260, 400)
    np.testing.assert_allclose(s.entries(qi, qj), want[qi, qj], rtol=1e-10,
                               atol=1e-11 * float(np.abs(want).max()))
    ti, tj, _ = s.topk(16)
    from compmatmul_b200.planted import topk_dense_host
    wi, wj, _ = topk_dense_host(want, 16)
    assert set(zip(ti.tolist(), tj.tolist())) == set(zip(wi.tolist(), wj.tolist()))


@pytest.mark.gpu
def test_sketch_topk_ties_across_tiles(gpu):
    import torch
    # all-zero inputs: every estimate is +-0; ties resolve as in the dense top-K
    AT = torch.zeros((16, 50), dtype=torch.float64, device="cuda")
    B = torch.zeros((16, 40), dtype=torch.float64, device="cuda")
    s = Sketch.compute(AT, B, 3, 256, 1, "fwht")
    ti, tj, tv = s.topk(100, scratch_bytes=8 * 40 * 7)
    di, dj, dv = device.topk(s.dense(), 100)
    np.testing.assert_array_equal(ti, di)  # (+0 before -0, then (i, j) order), as the dense path
    np.testing.assert_array_equal(tj, dj)
    assert np.all(tv == 0.0)
