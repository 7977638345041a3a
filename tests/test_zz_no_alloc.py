"""The no-allocation log-likelihood entry point, through the C ABI.

`gpum_b200_loglik_batch_noalloc` serves callers that cannot allocate device
memory (their device memory belongs to another allocator or a fixed budget):
they pass their own device buffers, and the library's scratch is a fixed
16 MiB __device__ array.  It must agree with the allocating entry point
(`gpum_b200_loglik_batch`) to the tolerance the other evaluation tests use
(1e-6 relative on the summed log-likelihood), on consecutive calls that reuse
the same scratch.  The test owns (allocates) the buffers, as such a caller
would; the entry point itself allocates nothing.
"""
import ctypes as C

import numpy as np
import pytest

from gpumetropolis_b200 import workloads as W

pytestmark = pytest.mark.gpu

REL_SUM = 1e-6


def _device_layout(torch, data, n_obs, n_cols):
    ld = (n_obs + 3) // 4 * 4
    cols = torch.zeros((n_cols, ld), dtype=torch.float32, device="cuda")
    cols[:, :n_obs] = torch.from_numpy(np.ascontiguousarray(data.T, dtype=np.float32)).cuda()
    return cols, ld


def _noalloc(native, m, cols, ld, n_obs, pts_dev, out_dev, stream):
    lib = native.load()
    code = np.ascontiguousarray(m.loglik.code, dtype=np.uint32)
    consts = np.ascontiguousarray(m.loglik.consts, dtype=np.float64)
    err = C.create_string_buffer(1024)
    rc = lib.gpum_b200_loglik_batch_noalloc(
        code.ctypes.data_as(C.POINTER(C.c_uint32)), code.size,
        consts.ctypes.data_as(C.POINTER(C.c_double)), consts.size, m.n_params,
        C.c_void_p(cols.data_ptr()), ld, m.n_cols, n_obs, C.c_void_p(pts_dev.data_ptr()),
        pts_dev.shape[0], C.c_void_p(out_dev.data_ptr()), C.c_void_p(stream), err, 1024)
    return rc, err.value.decode()


@pytest.mark.parametrize("name,n_obs", [("logistic", 4099), ("mixture", 20011)])
def test_noalloc_matches_allocating_entry_point(gpu, name, n_obs):
    torch = pytest.importorskip("torch")
    w = W.make(name, n_obs=n_obs)
    m = w.model
    cols, ld = _device_layout(torch, w.data, w.n_obs, m.n_cols)
    stream = torch.cuda.current_stream().cuda_stream
    base = np.zeros(m.n_params)
    if name == "logistic":
        base[:] = w.truth["beta"]
    else:
        base[:] = [np.log(0.3 / 0.7), -2.0, 3.0, 0.0, np.log(1.5)]
    # two consecutive calls with different batches share the scratch array
    for n_points, seed in ((37, 1), (301, 2)):
        pts = base + np.random.default_rng(seed).normal(0, 0.05, (n_points, m.n_params))
        pts_dev = torch.from_numpy(pts).cuda()
        out_dev = torch.full((n_points,), float("nan"), dtype=torch.float64, device="cuda")
        rc, msg = _noalloc(gpu, m, cols, ld, w.n_obs, pts_dev, out_dev, stream)
        assert rc == gpu.OK, msg
        got = out_dev.cpu().numpy()
        ref = gpu.loglik_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols,
                               w.n_obs, pts)
        rel = np.abs(got - ref) / np.abs(ref)
        assert rel.max() <= REL_SUM, (n_points, rel.max())


def test_noalloc_rejects_what_does_not_fit(gpu):
    torch = pytest.importorskip("torch")
    w = W.make("logistic", n_obs=512)
    m = w.model
    cols, ld = _device_layout(torch, w.data, w.n_obs, m.n_cols)
    stream = torch.cuda.current_stream().cuda_stream
    # 17 params x 300k points of f32 parameters alone exceed the 16 MiB scratch
    pts_dev = torch.zeros((300_000, m.n_params), dtype=torch.float64, device="cuda")
    out_dev = torch.zeros(300_000, dtype=torch.float64, device="cuda")
    rc, msg = _noalloc(gpu, m, cols, ld, w.n_obs, pts_dev, out_dev, stream)
    assert rc == gpu.ERR_UNSUPPORTED and "scratch" in msg
    # a misaligned leading dimension is refused before any launch
    rc, msg = _noalloc(gpu, m, cols, ld + 1, w.n_obs, pts_dev[:4], out_dev[:4], stream)
    assert rc == gpu.ERR_INVALID
