"""outputFusionCPU's CASE debug outputs (stereo_mapper.cpp:628-719) through pm_output_case,
against the oracle: CASE 0 is the argmin of the plane-sweep cost, CASE 1 the argmin of the SGM
sum, both bit-exact against oracle/imgproc.case_argmin on the FP32 oracle's volumes (the same op
order as the kernels); CASE 2 is pm_output.  The FP16 form's CASE 0 is checked against the
argmin of its own FP16 cost volume plus its per-pixel offsets."""
import numpy as np
import pytest

import oracle
from oracle import imgproc as oip
from probabilistic_mapping_b200 import _lib, scene
from probabilistic_mapping_b200.mapper import StereoMapper

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def setup(W, H, D, S, paths, mode, precision=0, seed=41):
    fs = scene.make_frameset(W, H, 0.8 * W, S, seed=seed)
    rho0, drho = scene.plane_range(D)
    prm = dict(rho0=rho0, intensity_scale=1 / 255, num_paths=paths, p1=0.003, p2=0.01, tau_so=3.5 / 255,
               uniqueness_ratio=0.95, cost_mode=mode, precision=precision)
    m = StereoMapper(W, H, D, **prm)
    m.initIntrinsic(fs.K, 0.0, drho)
    o = oracle.Mapper(oracle.Params(W=W, H=H, D=D, drho=drho, rho0=rho0, intensity_scale=1 / 255, cost_mode=mode,
                                    num_paths=paths, p1=0.003, p2=0.01, tau_so=3.5 / 255, uniqueness=0.95), fs.K,
                      prec="f32")
    m.initReference(fs.ref)
    o.init_reference(fs.ref)
    for s in range(S):
        m.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
        o.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
    return m, o, rho0, drho


@pytest.mark.parametrize("mode,paths,D", [(0, 4, 64), (1, 8, 64), (0, 8, 96)])
def test_case_outputs_match_oracle(mode, paths, D):
    W, H, S = 128, 96, 3
    m, o, rho0, drho = setup(W, H, D, S, paths, mode)
    st = o.stages()
    for case, vol in ((0, st["cost"]), (1, st["sgm"])):
        got = m.outputCase(case)
        want, widx = oip.case_argmin(vol.reshape(H, W, D), rho0, drho)
        assert (got.view(np.uint32) == want.view(np.uint32)).all(), case
        assert (m.wta_index() == widx).all(), case
    assert (got != 0).any() and (got != 10000).any()
    assert (m.outputCase(0) == 10000).any()        # border pixels no source sees
    np.testing.assert_array_equal(m.outputCase(2), m.output())
    np.testing.assert_array_equal(m.output().view(np.uint32), st["depth"].view(np.uint32))
    with pytest.raises(_lib.PmError):
        m.outputCase(3)
    m.close()


def test_case0_fp16_volume():
    W, H, D, S = 128, 96, 64, 3
    m, _, rho0, drho = setup(W, H, D, S, 4, 0, precision=_lib.PM_PREC_FP16)
    got = m.outputCase(0)
    from cuda.bindings import runtime as rt
    b = m.buffers()
    vol = torch.empty(H * W * D, dtype=torch.float16, device="cuda")
    torch.cuda.synchronize()
    off = torch.empty(H * W, dtype=torch.float32, device="cuda")
    err, = rt.cudaMemcpy(vol.data_ptr(), b.cost, vol.numel() * 2, rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
    assert err == rt.cudaError_t.cudaSuccess
    err, = rt.cudaMemcpy(off.data_ptr(), b.cost_offset, off.numel() * 4, rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
    assert err == rt.cudaError_t.cudaSuccess
    # the half volume holds cost - offset[pixel]; the kernel adds it back in FP32
    full = vol.float().reshape(H * W, D) + off[:, None]
    want, _ = oip.case_argmin(full.cpu().numpy().reshape(H, W, D), rho0, drho)
    assert (got.view(np.uint32) == want.view(np.uint32)).all()
    m.close()
