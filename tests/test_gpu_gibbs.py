"""Gibbs penalties on the GPU (gibbs.cu through the C ABI) against the oracle's restatement of GibbsPenalty.inl."""
import zlib

import numpy as np
import pytest

from stir_b200 import _abi

pytestmark = pytest.mark.gpu

TEST_PACK_WEIGHTS = np.array([[[0, 1, 0], [1, 0, 1], [0, 1, 0]]], np.float32)  # OSMAPOSL_test_PM_QPweights.par


def _weights(kind):
    if kind is None:
        return None
    if kind == "test_pack":
        return TEST_PACK_WEIGHTS
    if kind == "even":  # 2x4x3: STIR appends (in effect) a zero plane / row
        return np.random.default_rng(6).uniform(0, 1, (2, 4, 3)).astype(np.float32)
    w = np.random.default_rng(5).uniform(0, 1, (5, 3, 7)).astype(np.float32)
    w = (w + w[::-1, ::-1, ::-1]) / 2
    w[2, 1, 3] = 0
    return np.ascontiguousarray(w, np.float32)


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


def _make(cls, weights, only_2D, beta, shape, vox, layout, kappa):
    from stir_b200 import gibbs
    p = cls(only_2D=only_2D, penalisation_factor=beta) if cls is gibbs.GibbsQuadraticPenalty else \
        cls(only_2D=only_2D, penalisation_factor=beta, gamma=2.0, epsilon=0.01)
    if weights is not None:
        p.set_weights(weights)
    if kappa is not None:
        p.set_kappa_sptr(kappa)
    p.set_up(shape, vox, layout)
    return p


@pytest.mark.parametrize("potential", ["quadratic", "rdp"])
@pytest.mark.parametrize("weights", [None, "2D", "test_pack", "5x3x7", "even"])
@pytest.mark.parametrize("layout", [_abi.LAYOUT_STIR, _abi.LAYOUT_DEVICE])
@pytest.mark.parametrize("with_kappa", [False, True])
def test_gibbs_matches_oracle(cuda_device, oracle_lib, potential, weights, layout, with_kappa):
    import torch
    from stir_b200 import gibbs
    O = oracle_lib
    cls = gibbs.GibbsQuadraticPenalty if potential == "quadratic" else gibbs.GibbsRelativeDifferencePenalty
    pot = 1 if potential == "quadratic" else 2
    shape, vox, beta = (9, 11, 13), (2.0, 3.0, 3.0), 0.7
    rng = np.random.default_rng(zlib.crc32(repr((potential, weights, layout, with_kappa)).encode()))
    x = rng.uniform(0.2, 2.0, shape).astype(np.float32)
    v = rng.uniform(-1.0, 1.0, shape).astype(np.float32)
    kappa = rng.uniform(0.5, 1.5, shape).astype(np.float32) if with_kappa else None
    only_2D = weights == "2D"
    w = _weights(None if only_2D else weights)
    wo = w if w is not None else O.gibbs_default_weights(vox, only_2D=only_2D)

    def dev(a):  # host [z][y][x] -> device tensor in `layout`
        t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        return t if layout == _abi.LAYOUT_STIR else t.permute(1, 2, 0).contiguous().view(-1)

    def host(t):
        t = t.cpu()
        return t.numpy() if layout == _abi.LAYOUT_STIR else t.view(shape[1], shape[2], shape[0]).permute(2, 0, 1).numpy()

    kd = dev(kappa) if kappa is not None else None
    p = _make(cls, w, only_2D, beta, shape, vox, layout, kd)
    assert np.array_equal(p.get_weights(), wo)
    xd, vd = dev(x), dev(v)
    args = dict(kappa=kappa, gamma=2.0, epsilon=0.01)
    ref_v = O.gibbs("value", pot, beta, wo, x, **args)
    assert abs(p.compute_value(xd) - ref_v) <= 1e-12 * abs(ref_v)
    assert _rel(host(p.compute_gradient(xd)), O.gibbs("gradient", pot, beta, wo, x, **args)) <= 1e-7
    ref_gti = O.gibbs("gradient_times_input", pot, beta, wo, x, input_image=v, **args)
    assert abs(p.compute_gradient_times_input(vd, xd) - ref_gti) <= 1e-12 * max(abs(ref_gti), 1.0)
    assert _rel(host(p.compute_Hessian_diagonal(xd)), O.gibbs("hessian_diagonal", pot, beta, wo, x, **args)) <= 1e-7
    base = rng.uniform(-1, 1, shape).astype(np.float32)
    out = dev(base)
    p.accumulate_Hessian_times_input(out, xd, vd)
    ref = O.gibbs("hessian_times_input", pot, beta, wo, x, input_image=v, out=base, **args)
    assert _rel(host(out), ref) <= 1e-6
    for voxel in [(0, 0, 0), (4, 5, 6), (8, 10, 12)]:
        hd = host(p.compute_Hessian(voxel, xd))
        assert _rel(hd, O.gibbs("hessian", pot, beta, wo, x, voxel=voxel, **args)) <= 1e-6


def test_gibbs_clinical_image_and_errors(cuda_device, oracle_lib):
    """The clinical image size (344x344x127, device layout): gradient against the oracle; a zero penalisation
    factor; STIR's errors before set-up and for an image of another size."""
    import torch
    from stir_b200 import gibbs
    O = oracle_lib
    shape, vox = (127, 344, 344), (2.03, 2.09, 2.09)
    x = torch.rand(shape, device="cuda") + 0.1
    p = gibbs.GibbsRelativeDifferencePenalty(penalisation_factor=0.1, gamma=2.0, epsilon=1e-7)
    with pytest.raises(RuntimeError):
        p.compute_value(x)
    p.set_up(shape, vox)
    g = p.compute_gradient(x).cpu().numpy()
    xs = x.cpu().numpy()
    ref = O.gibbs("gradient", 2, 0.1, O.gibbs_default_weights(vox), xs, gamma=2.0, epsilon=1e-7)
    assert _rel(g, ref) <= 1e-7
    with pytest.raises(ValueError):
        p.compute_gradient(torch.rand((10, 10, 10), device="cuda"))
    z = gibbs.GibbsQuadraticPenalty(penalisation_factor=0.0)
    z.set_up(shape, vox)
    assert z.compute_value(x) == 0.0
    assert not z.compute_gradient(x).any()
    bad = gibbs.GibbsQuadraticPenalty(penalisation_factor=1.0)
    with pytest.raises(ValueError):
        bad.set_weights(np.ones((9, 3, 3), np.float32))


def _ref_cuda(oracle_lib):
    if not oracle_lib.ref_cuda_priors_available():
        pytest.skip("STIR's CUDA prior kernels were not built (oracle/_ref needs the STIR sources)")
    return oracle_lib.ref_cuda_priors()


@pytest.mark.parametrize("potential", ["quadratic", "rdp"])
@pytest.mark.parametrize("with_kappa", [False, True])
@pytest.mark.parametrize("layout", [_abi.LAYOUT_STIR, _abi.LAYOUT_DEVICE])
def test_cuda_arithmetic_gradient_equals_stirs_cuda_kernel(cuda_device, oracle_lib, potential, with_kappa, layout):
    """CudaGibbs*Penalty's gradient (float sums) against STIR's own CudaGibbsPenalty_gradient_kernel built for this
    GPU (oracle/_ref), on the same device image with the default 3x3x3 weights: equal bit for bit; and within float
    rounding of the host arithmetic (double sums, the oracle)."""
    import ctypes
    import torch
    from stir_b200 import gibbs
    ref = _ref_cuda(oracle_lib)
    shape, vox, beta = (23, 37, 41), (2.03, 2.09, 2.09), 0.3
    rng = np.random.default_rng(11 + with_kappa)
    x = torch.from_numpy(rng.uniform(0.0, 3.0, shape).astype(np.float32)).cuda()
    x[3:5] = 0.0  # zero voxels: the Relative Difference potential's special case
    kappa = torch.from_numpy(rng.uniform(0.5, 1.5, shape).astype(np.float32)).cuda() if with_kappa else None
    cls = gibbs.CudaGibbsQuadraticPenalty if potential == "quadratic" else gibbs.CudaGibbsRelativeDifferencePenalty
    p = cls(penalisation_factor=beta) if potential == "quadratic" else cls(penalisation_factor=beta, gamma=2.0,
                                                                            epsilon=1e-7)

    def to_layout(t):  # [z][y][x] -> the penalty's layout
        return t if layout == _abi.LAYOUT_STIR else t.permute(1, 2, 0).contiguous()

    def from_layout(t):
        return t if layout == _abi.LAYOUT_STIR else t.view(shape[1], shape[2], shape[0]).permute(2, 0, 1).contiguous()

    if kappa is not None:
        p.set_kappa_sptr(to_layout(kappa))
    p.set_up(shape, vox, layout)
    got = from_layout(p.compute_gradient(to_layout(x)))
    w = torch.from_numpy(np.ascontiguousarray(p.get_weights(), np.float32)).cuda()
    out = torch.full(shape, float("nan"), device="cuda")
    st = ref.ref_cuda_gibbs_gradient(1 if potential == "rdp" else 0, ctypes.c_void_p(out.data_ptr()),
                                     ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(w.data_ptr()), 3, 3, 3,
                                     None if kappa is None else ctypes.c_void_p(kappa.data_ptr()), beta, 2.0, 1e-7,
                                     shape[0], shape[1], shape[2], -(shape[1] // 2), -(shape[2] // 2),
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    torch.cuda.synchronize()
    assert torch.equal(got, out), float((got - out).abs().max())
    host = gibbs.GibbsRelativeDifferencePenalty(penalisation_factor=beta, gamma=2.0, epsilon=1e-7) \
        if potential == "rdp" else gibbs.GibbsQuadraticPenalty(penalisation_factor=beta)
    if kappa is not None:
        host.set_kappa_sptr(kappa)
    host.set_up(shape, vox)
    assert _rel(got.cpu().numpy(), host.compute_gradient(x).cpu().numpy()) <= 1e-6


def test_stirs_cuda_rdp_prior_kernel_matches_oracle(cuda_device, oracle_lib):
    """STIR's CudaRelativeDifferencePrior gradient kernel (built for this GPU) against the oracle's
    RelativeDifferencePrior gradient: both sum in double, so they agree to float rounding."""
    import ctypes
    import torch
    from stir_b200 import _abi as A
    ref = _ref_cuda(oracle_lib)
    shape, vox = (17, 29, 31), (2.03, 2.09, 2.09)
    x = torch.from_numpy(np.random.default_rng(3).uniform(0.1, 3.0, shape).astype(np.float32)).cuda()
    w = torch.from_numpy(np.ascontiguousarray(oracle_lib.gibbs_default_weights(vox), np.float32)).cuda()
    out = torch.zeros(shape, device="cuda")
    st = ref.ref_cuda_rdp_prior_gradient(ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                         ctypes.c_void_p(w.data_ptr()), None, 2.0, 0.01, 0.5, *shape,
                                         ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    torch.cuda.synchronize()
    pr = A.Prior(type=A.PRIOR_RELATIVE_DIFFERENCE, penalisation_factor=0.5, gamma=2.0, epsilon=0.01, only_2D=0,
                 map_model=A.MAP_MULTIPLICATIVE, kappa_dev=None)
    assert _rel(out.cpu().numpy(), oracle_lib.prior_gradient(pr, x.cpu().numpy(), vox)) <= 1e-6
