"""The no-allocation log-likelihood entry point, through the C ABI.

`gpum_b200_loglik_batch_noalloc` serves callers that cannot allocate device
memory (their device memory belongs to another allocator or a fixed budget):
they pass their own device buffers, and the library's scratch is a fixed
16 MiB __device__ array.  It must agree with the allocating entry point
(`gpum_b200_loglik_batch`) and with the f64 oracle to the tolerance the other
evaluation tests use (1e-6 relative on the summed log-likelihood), on
consecutive calls that reuse the same scratch with different shapes.  The
test owns (allocates) the buffers, as such a caller would; the entry point
itself allocates nothing, which the device's free memory before and after a
call confirms.
"""
import ctypes as C

import numpy as np
import pytest

from gpumetropolis_b200 import workloads as W
from gpumetropolis_b200.dsl import gpum_model
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL_SUM = 1e-6


def _device_layout(torch, data, n_obs, n_cols):
    ld = (n_obs + 3) // 4 * 4
    cols = torch.zeros((max(n_cols, 1), ld), dtype=torch.float32, device="cuda")
    if n_cols:
        cols[:, :n_obs] = torch.from_numpy(np.ascontiguousarray(data.T, dtype=np.float32)).cuda()
    return cols, ld


def _noalloc(native, code, consts, n_params, cols, ld, n_cols, n_obs, pts_dev, out_dev,
             stream):
    lib = native.load()
    code = np.ascontiguousarray(code, dtype=np.uint32)
    consts = np.ascontiguousarray(consts, dtype=np.float64)
    err = C.create_string_buffer(1024)
    rc = lib.gpum_b200_loglik_batch_noalloc(
        code.ctypes.data_as(C.POINTER(C.c_uint32)), code.size,
        consts.ctypes.data_as(C.POINTER(C.c_double)), consts.size, n_params,
        C.c_void_p(cols.data_ptr() if cols is not None else 0), ld, n_cols, n_obs,
        C.c_void_p(pts_dev.data_ptr()), pts_dev.shape[0], C.c_void_p(out_dev.data_ptr()),
        C.c_void_p(stream), err, 1024)
    return rc, err.value.decode()


def _check(gpu, torch, code, consts, n_params, data, n_cols, n_obs, cols, ld, pts, stream):
    pts_dev = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
    out_dev = torch.full((pts.shape[0],), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rc, msg = _noalloc(gpu, code, consts, n_params, cols, ld, n_cols, n_obs, pts_dev, out_dev,
                       stream)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert rc == gpu.OK, msg
    got = out_dev.cpu().numpy()
    ref = O.loglik_batch(code, consts, n_params, data, n_cols, n_obs, pts)
    rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)
    assert rel.max() <= REL_SUM, rel.max()
    return got, ref, free0, free1


@pytest.mark.parametrize("name,n_obs", [("logistic", 4099), ("mixture", 20011)])
def test_noalloc_matches_both_entry_points(gpu, name, n_obs):
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
    # two consecutive calls with different batches share the scratch array;
    # the first call of the process may place the 16 MiB array (the library's
    # device code loads lazily), every later one must leave free memory as is
    for k, (n_points, seed) in enumerate(((37, 1), (301, 2), (64, 3))):
        pts = base + np.random.default_rng(seed).normal(0, 0.05, (n_points, m.n_params))
        got, _, free0, free1 = _check(gpu, torch, m.loglik.code, m.loglik.consts, m.n_params,
                                      w.data, m.n_cols, w.n_obs, cols, ld, pts, stream)
        if k > 0:
            assert free1 == free0  # the call allocated no device memory
        alloc = gpu.loglik_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols,
                                 w.n_obs, pts)
        rel = np.abs(got - alloc) / np.abs(alloc)
        assert rel.max() <= REL_SUM, (n_points, rel.max())


def test_noalloc_deep_programs_and_shapes_in_a_row(gpu):
    # Stack depths 3, 12 and 24 take the three interpreter variants (8, 4 and
    # 2 chains per thread); the calls alternate parameter counts and batch
    # sizes, so each one reuses scratch the previous one left with another
    # layout.  Then a program that reads no data column (n_cols = 0): its
    # per-observation term still counts once per observation.
    torch = pytest.importorskip("torch")
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(3)
    n_obs = 3001
    # positive data and parameters: every term positive, so the sums do not
    # cancel and the relative bound applies as stated
    y = rng.uniform(0.5, 1.5, n_obs)
    cols, ld = _device_layout(torch, y.reshape(-1, 1), n_obs, 1)
    for depth, n_points in ((12, 50), (24, 7), (3, 129), (24, 400)):
        f = "~ " + "(y * a + " * (depth - 1) + "b" + ")" * (depth - 1)
        m = gpum_model(f, ["a", "b"], "y")
        assert gpu.validate_program(m.loglik.code, m.loglik.consts.size, 2, 1) >= depth
        pts = rng.uniform(0.1, 0.5, (n_points, 2))
        _check(gpu, torch, m.loglik.code, m.loglik.consts, 2, y.reshape(-1, 1), 1, n_obs,
               cols, ld, pts, stream)
    w = W.make("logistic", n_obs=2048)
    lc, lld = _device_layout(torch, w.data, w.n_obs, w.model.n_cols)
    pts = w.truth["beta"] + rng.normal(0, 0.05, (64, w.model.n_params))
    _check(gpu, torch, w.model.loglik.code, w.model.loglik.consts, w.model.n_params, w.data,
           w.model.n_cols, w.n_obs, lc, lld, pts, stream)
    m0 = gpum_model("~ log(mu) - mu", "mu", [])
    assert m0.n_cols == 0
    pts = rng.uniform(0.5, 2.0, (33, 1))
    got, ref, _, _ = _check(gpu, torch, m0.loglik.code, m0.loglik.consts, 1,
                            np.zeros((n_obs, 0)), 0, n_obs, None, 0, pts, stream)
    np.testing.assert_allclose(ref, n_obs * (np.log(pts[:, 0]) - pts[:, 0]), rtol=1e-12)


def test_noalloc_rejects_what_does_not_fit(gpu):
    torch = pytest.importorskip("torch")
    w = W.make("logistic", n_obs=512)
    m = w.model
    cols, ld = _device_layout(torch, w.data, w.n_obs, m.n_cols)
    stream = torch.cuda.current_stream().cuda_stream
    # 17 params x 300k points of f32 parameters alone exceed the 16 MiB scratch
    pts_dev = torch.zeros((300_000, m.n_params), dtype=torch.float64, device="cuda")
    out_dev = torch.zeros(300_000, dtype=torch.float64, device="cuda")
    rc, msg = _noalloc(gpu, m.loglik.code, m.loglik.consts, m.n_params, cols, ld, m.n_cols,
                       w.n_obs, pts_dev, out_dev, stream)
    assert rc == gpu.ERR_UNSUPPORTED and "scratch" in msg
    # a misaligned leading dimension is refused before any launch
    rc, msg = _noalloc(gpu, m.loglik.code, m.loglik.consts, m.n_params, cols, ld + 1, m.n_cols,
                       w.n_obs, pts_dev[:4], out_dev[:4], stream)
    assert rc == gpu.ERR_INVALID
