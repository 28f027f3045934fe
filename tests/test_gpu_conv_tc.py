"""GPU tests of the guess network's tensor-core convolution (ewg_net_conv3d: tcgen05.mma into tensor
memory with TMA loads of the shifted input boxes, k_conv3d_tc) against an FP64 NumPy convolution of
the same BF16 inputs and weights. Bound: every output within 2^-8 of its own magnitude plus 1e-5 of
the layer's output scale (the BF16 rounding of an FP32 sum of at most 864 products). Covered: both
input widths (16 and 32 channels), both epilogues (bias + ReLU, ReLU mask of the layer below), and
volumes whose x / y extents are not multiples of the 32 x 4 voxel tile, where the TMA boxes reach past
the volume and the convolution's zero padding is the copy's zero fill; volumes at least 96 wide, which
take the ring kernel (rows of 128 voxels in segments of 16 rows, each input row loaded once per segment
into a ring and shared by three output rows), with and without a partial last row tile, with several
segments per column and a last segment of one row; a batch of two volumes checks that no tap reads
across volumes."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bf16_bits(a):
    """float -> bfloat16 bit patterns (round to nearest even)."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def _from_bits(b):
    return (b.astype(np.uint32) << 16).view(np.float32)


def _reference(x, w, bias, mask, epilogue):
    """x [B, D, H, W, C], w [27, 32, C] (tap = 9 (dz + 1) + 3 (dy + 1) + dx + 1), FP64."""
    B, D, H, W, Cc = x.shape
    xp = np.zeros((B, D + 2, H + 2, W + 2, Cc))
    xp[:, 1:-1, 1:-1, 1:-1] = x
    acc = np.zeros((B, D, H, W, w.shape[1]))
    for t in range(27):
        dx, dy, dz = t % 3 - 1, (t // 3) % 3 - 1, t // 9 - 1
        acc += xp[:, 1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :] @ w[t].T
    if epilogue == 0:
        return np.maximum(acc + bias, 0.0)
    return acc * (mask > 0)


def _conv(lib, torch, cin, epilogue, shape, seed):
    rng = np.random.default_rng(seed)
    B, D, H, W = shape
    x = _bf16_bits(rng.normal(size=(B, D, H, W, cin)))
    w = _bf16_bits(rng.normal(0, 1 / np.sqrt(27 * cin), size=(27, 32, cin)))
    bias = rng.normal(0, 0.1, size=32).astype(np.float32)
    mask = _bf16_bits(rng.normal(size=(B, D, H, W, 32)))
    dev = "cuda"
    tx = torch.from_numpy(x.view(np.int16)).to(dev)
    tw = torch.from_numpy(w.view(np.int16)).to(dev)
    tb = torch.from_numpy(bias).to(dev)
    tm = torch.from_numpy(mask.view(np.int16)).to(dev)
    ty = torch.full((B * D * H * W * 32,), -1, dtype=torch.int16, device=dev)
    st = lib.ewg_net_conv3d(cin, epilogue, B, D, H, W, C.c_void_p(tx.data_ptr()), C.c_void_p(tw.data_ptr()),
                            C.c_void_p(tb.data_ptr()), C.c_void_p(tm.data_ptr()), C.c_void_p(ty.data_ptr()),
                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, st
    y = _from_bits(ty.cpu().numpy().view(np.uint16)).reshape(B, D, H, W, 32).astype(np.float64)
    ref = _reference(_from_bits(x).astype(np.float64), _from_bits(w).astype(np.float64), bias.astype(np.float64),
                     _from_bits(mask), epilogue)
    return y, ref


@pytest.mark.parametrize("cin", [16, 32])
@pytest.mark.parametrize("epilogue", [0, 2])
@pytest.mark.parametrize("shape", [(1, 4, 8, 32), (1, 3, 5, 40), (2, 4, 7, 33), (1, 3, 5, 130), (2, 2, 3, 128),
                                   (1, 2, 4, 200), (1, 2, 19, 100), (2, 1, 17, 128), (1, 3, 33, 96)])
def test_tensor_core_conv_matches_fp64(ewg_mod, cin, epilogue, shape):
    import torch
    lib = ewg_mod.load()
    fn = lib.ewg_net_conv3d
    fn.restype = C.c_int
    fn.argtypes = [C.c_int32] * 6 + [C.c_void_p] * 6
    y, ref = _conv(lib, torch, cin, epilogue, shape, seed=cin + 7 * epilogue + sum(shape))
    scale = np.max(np.abs(ref))
    err = np.abs(y - ref)
    bound = 2.0 ** -8 * np.abs(ref) + 1e-5 * scale
    assert np.all(err <= bound), (float(np.max(err / (np.abs(ref) + 1e-5 * scale))), scale)
    assert scale > 0.1


def test_tensor_core_conv_rejects_bad_arguments(ewg_mod):
    lib = ewg_mod.load()
    fn = lib.ewg_net_conv3d
    fn.restype = C.c_int
    fn.argtypes = [C.c_int32] * 6 + [C.c_void_p] * 6
    import torch
    buf = torch.zeros(64 * 32, dtype=torch.int16, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    assert fn(24, 0, 1, 1, 1, 1, p, p, p, p, p, None) == ewg_mod.EWG_ERR_INVALID        # channels
    assert fn(32, 1, 1, 1, 1, 1, p, p, p, p, p, None) == ewg_mod.EWG_ERR_INVALID        # epilogue
    assert fn(32, 0, 1, 0, 1, 1, p, p, p, p, p, None) == ewg_mod.EWG_ERR_INVALID        # extent
    assert fn(32, 0, 1, 1, 1, 1, C.c_void_p(buf.data_ptr() + 2), p, p, p, p, None) == ewg_mod.EWG_ERR_INVALID
