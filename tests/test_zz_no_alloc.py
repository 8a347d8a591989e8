"""GPU test of the allocation-free FP32 AR filter entry point.

``arma_ar_filter_fp32c_noalloc`` is for callers that cannot allocate device
memory where they filter a surface (code running inside another framework's
memory pool, allocation-free serving loops, plugins whose host process owns
the device allocator).  It keeps all of its scratch in one static device
array.  This test calls it twice in a row through the C ABI on the same noise
and checks each result against the context-based ``arma_ar_filter`` (FP32C),
which builds the same coefficient tables and runs the same kernel, so the
two must agree bit for bit, and against the FP64 oracle filter on the same
noise within the FP32 filter's test tolerance (RMS <= 1e-5 relative).  It
also checks that oversized requests and a capturing stream are refused.  It
lives in its own file, collected last, and passes alone in a fresh process as
well as after the other tests.
"""
import numpy as np
import pytest

import arma_b200 as A
from arma_b200 import capi
import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def rms_rel(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    return np.sqrt(np.mean((a - b) ** 2) / np.mean(b * b))


def _model(kind, order):
    if kind == A.ACF_STANDING:
        return A.ar_fit_analytic(kind, order, 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    return A.ar_fit_analytic(kind, order, 1.0, 0.6, [0.04] * 3, [0.3, 0.2])


@pytest.mark.parametrize("shape,order,kind", [
    ((40, 50, 70), (4, 6, 8), A.ACF_STANDING),
    ((48, 64, 40), (10, 10, 10), A.ACF_PROPAGATING),
    ((40, 20, 40), (16, 1, 1), A.ACF_STANDING),  # the longest time order accepted
])
def test_noalloc_matches_context_filter_twice(ctx, shape, order, kind):
    phi, var = _model(kind, order)
    eps = O.white_noise(O.mt19937_params(), 21, np.sqrt(var), int(np.prod(shape)))
    eps = eps.reshape(shape)
    eps32 = eps.astype(np.float32)
    fp64 = O.ar_filter(eps32.astype(np.float64), phi)  # FP64 oracle on the same noise

    ref = torch.as_tensor(eps32).cuda()
    ctx.ar_filter(phi, shape, A.FP32C, ref.data_ptr())
    ctx.synchronize()
    expected = ref.cpu().numpy()

    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # two calls in a row share the static scratch
        z = torch.as_tensor(eps32).cuda()
        torch.cuda.synchronize()
        capi.ar_filter_fp32c_noalloc(stream, phi, shape, z.data_ptr())
        got = z.cpu().numpy()
        assert np.isfinite(got).all()
        assert np.array_equal(got, expected)
        assert rms_rel(got, fp64) <= 1e-5


def test_noalloc_rejects_oversized_request():
    phi = np.zeros((13, 13, 13))  # 2197 coefficients > 2048
    z = torch.zeros((2, 16, 32), dtype=torch.float32, device="cuda")
    with pytest.raises(capi.ArmaError) as e:
        capi.ar_filter_fp32c_noalloc(0, phi, z.shape, z.data_ptr())
    assert e.value.code == -1 and "2048" in str(e.value)
    big = (2, 16 * 128, 32 * 65)  # 128 x 65 = 8320 tiles > 8192
    with pytest.raises(capi.ArmaError) as e:
        capi.ar_filter_fp32c_noalloc(0, np.zeros((2, 2, 2)), big, z.data_ptr())
    assert e.value.code == -1 and "8192" in str(e.value)
    with pytest.raises(capi.ArmaError) as e:  # above 16 per axis
        capi.ar_filter_fp32c_noalloc(0, np.zeros((17, 1, 1)), z.shape, z.data_ptr())
    assert e.value.code == -8


def test_noalloc_refuses_a_capturing_stream():
    """The call synchronises its stream, so it cannot be recorded into a CUDA
    graph; a capturing stream is refused before any device work."""
    phi, _ = _model(A.ACF_STANDING, (2, 2, 2))
    z = torch.zeros((4, 16, 32), dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        g.capture_begin()
        try:
            with pytest.raises(capi.ArmaError) as e:
                capi.ar_filter_fp32c_noalloc(s.cuda_stream, phi, z.shape, z.data_ptr())
        finally:
            z.add_(0.0)  # give the captured graph one node
            g.capture_end()
    assert e.value.code == -1 and "capturing" in str(e.value)
    g.reset()
