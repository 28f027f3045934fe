"""GPU test of ewg_net_forward_noalloc, the guess network's forward pass that allocates nothing
and keeps its activations in a fixed device array shared by all calls.

Calls in a row, with different parameters and shapes (leftovers of an earlier call in the shared
array would show in a later one), the last at exactly EWG_NET_NOALLOC_MAX_VOXELS voxels where the
array's bounds are tightest, each checked against ewg_net_eval_host with the same parameters and
features. Both paths cast the features and weights to BF16 with the same rounding and run the same
convolution kernels, in which each output voxel is computed by one thread in a fixed order, so the
outputs must agree bit for bit. A batch above EWG_NET_NOALLOC_MAX_VOXELS is rejected with
EWG_ERR_INVALID and a message."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_VOXELS = 65536


def _params(ewg, rng, n_params):
    p = np.zeros(n_params, dtype=np.float32)
    for (w, b, ci, co), cir, cor in zip(ewg.net_layout(), ewg.NET_CIN_REAL, ewg.NET_COUT_REAL):
        W = np.zeros((27, co, ci), dtype=np.float32)
        W[:, :cor, :cir] = rng.normal(0, 0.9 / np.sqrt(27 * cir), size=(27, cor, cir))
        p[w:b] = W.ravel()
        p[b:b + cor] = rng.normal(0, 0.05, size=cor)
    return p


def _lib(ewg):
    lib = ewg.load()
    f = lib.ewg_net_forward_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_char_p, C.c_int32]
    return f


def _noalloc(fn, params, feat, shape):
    import torch
    B, D, H, W = shape
    dp = torch.from_numpy(params).cuda()
    df = torch.from_numpy(feat).cuda()
    out = torch.full((B, D, H, W, 2), float("nan"), dtype=torch.float32, device="cuda")
    msg = C.create_string_buffer(256)
    stream = torch.cuda.current_stream()
    st = fn(dp.data_ptr(), B, D, H, W, df.data_ptr(), out.data_ptr(), C.c_void_p(stream.cuda_stream), msg, 256)
    stream.synchronize()
    assert st == 0, msg.value.decode()
    return out.cpu().numpy()


def test_noalloc_forward_matches_eval_host(ewg_mod):
    fn = _lib(ewg_mod)
    rng = np.random.default_rng(11)
    net = ewg_mod.GuessNet(seed=2)
    for shape in ((2, 6, 7, 8), (1, 5, 9, 6), (1, 64, 64, 16)):
        assert np.prod(shape) <= MAX_VOXELS
        p = _params(ewg_mod, rng, net.n_params)
        net.set_params(p)
        f = rng.normal(size=shape + (5,)).astype(np.float32)
        y_ref, _, _ = net.eval_host(f)
        y = _noalloc(fn, p, f, shape)
        assert np.all(np.isfinite(y))
        assert np.array_equal(y, y_ref), (shape, float(np.max(np.abs(y - y_ref))))


def test_noalloc_rejects_batch_above_limit(ewg_mod):
    import torch
    fn = _lib(ewg_mod)
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    msg = C.create_string_buffer(256)
    # 1 x 64 x 64 x 17 = 69632 voxels > 65536; rejected before any pointer is read
    st = fn(dummy.data_ptr(), 1, 64, 64, 17, dummy.data_ptr(), dummy.data_ptr(), None, msg, 256)
    assert st == 1
    assert b"limit" in msg.value and str(MAX_VOXELS).encode() in msg.value
