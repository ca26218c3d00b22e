"""Backward kernels: adjoint dot-product test, FP64 finite differences, and
gradients against the pure-torch float64 reference (tests/torch_ref.py).

Tolerances: adjoint identity 1e-5 (relative, fp32 accumulation);
gradients vs float64 reference 2e-4 relative L2; finite differences
(central, h = 1e-4, float64 reference forward) 2e-3 relative per entry
against the GPU gradient (the interpolant is piecewise linear in the delay,
so entries whose perturbation crosses a sample boundary are skipped).
"""
import numpy as np
import pytest
import torch

import ffdas_b200
from ffdas_b200 import workloads as W
from ffdas_b200.autograd import das_autograd
from oracle import oracle
from tests.torch_ref import das_ref

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _problem(seed=0, B=2, C=6, S=3, N=128, nz=9, nx=7):
    g = torch.Generator().manual_seed(seed)
    x = torch.randn((B, C, S, N), generator=g)
    src = torch.zeros((C, 3))
    src[:, 0] = torch.linspace(-3, 3, C)
    zz, xx = torch.meshgrid(torch.linspace(20, 45, nz), torch.linspace(-4, 4, nx), indexing="ij")
    dst = torch.stack([xx, torch.zeros_like(xx), zz], -1)
    offs = torch.rand((S, nz, nx), generator=g) * 30 + 5
    w = torch.rand((S, nz, nx), generator=g) + 0.2
    return x, src, dst, offs, w


def test_adjoint_dot_product():
    x, src, dst, offs, w = (t.to(DEV) for t in _problem(1, B=3))
    xg = x.clone().requires_grad_(True)
    y = torch.randn((x.shape[0], *dst.shape[:-1]), device=DEV)
    out = das_autograd(xg, src, dst, offs, w)
    lhs = float((out.double() * y.double()).sum())
    (gx,) = torch.autograd.grad(out, xg, grad_outputs=y)
    rhs = float((x.double() * gx.double()).sum())
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), 1.0)


@pytest.mark.parametrize("B", [1, 2, 5])
def test_gradients_match_float64_reference(B):
    cpu = _problem(2, B=B)
    gpu = [t.to(DEV).requires_grad_(True) for t in cpu]
    ref = [t.double().requires_grad_(True) for t in cpu]
    g = torch.randn((B, *cpu[2].shape[:-1]), generator=torch.Generator().manual_seed(3))
    out = das_autograd(*gpu)
    out.backward(g.to(DEV))
    out_ref = das_ref(*ref)
    out_ref.backward(g.double())
    assert oracle.rel_l2(out.detach().cpu().numpy(), out_ref.detach().numpy()) < 2e-5
    for name, a, b in zip(["x", "srcpos", "dstpos", "offsets", "weights"], gpu, ref):
        err = oracle.rel_l2(a.grad.cpu().numpy(), b.grad.numpy())
        assert err < 2e-4, (name, err)


@pytest.mark.parametrize("B", [1, 4])
def test_autofocus_gradient_subset_matches_float64_reference(B):
    # the gradients an autofocus step takes (delays, voxel and channel
    # positions; x and the weights hold no grad), which the backward computes
    # without the channel-data scatter
    cpu = _problem(4, B=B)
    need = [False, True, True, True, False]
    gpu = [t.to(DEV).requires_grad_(n) for t, n in zip(cpu, need)]
    ref = [t.double().requires_grad_(n) for t, n in zip(cpu, need)]
    g = torch.randn((B, *cpu[2].shape[:-1]), generator=torch.Generator().manual_seed(5))
    das_autograd(*gpu).backward(g.to(DEV))
    das_ref(*ref).backward(g.double())
    for name, a, b, n in zip(["x", "srcpos", "dstpos", "offsets", "weights"], gpu, ref, need):
        if not n:
            assert a.grad is None, name
            continue
        err = oracle.rel_l2(a.grad.cpu().numpy(), b.grad.numpy())
        assert err < 2e-4, (name, err)


def test_sparse_gradients_match_reference():
    x, src, dst, offs, w = _problem(4, B=2, S=5)
    idx = torch.randint(0, 5, (3, *dst.shape[:-1]), generator=torch.Generator().manual_seed(5)).int()
    offs3, w3 = offs[:3].clone(), w[:3].clone()
    gpu = [t.to(DEV).requires_grad_(True) for t in (x, src, dst, offs3, w3)]
    ref = [t.double().requires_grad_(True) for t in (x, src, dst, offs3, w3)]
    out = ffdas_b200.das_sparse(*gpu, idx.to(DEV))
    out.sum().backward()
    das_ref(*ref, sparse_indices=idx).sum().backward()
    for name, a, b in zip(["x", "srcpos", "dstpos", "offsets", "weights"], gpu, ref):
        assert oracle.rel_l2(a.grad.cpu().numpy(), b.grad.numpy()) < 2e-4, name


@pytest.mark.parametrize("kernel", ["sorted", "gather"])
@pytest.mark.parametrize("C", [6, 128], ids=["one_slice", "channel_slices"])
@pytest.mark.parametrize("weights_grad", [True, False], ids=["all", "no_weight_grad"])
def test_sparse_gradients_uneven_lists(kernel, C, weights_grad):
    # uneven lists padded with zero weights, on the sorted-list adjoint (the
    # default: a lane per list entry) and the gather adjoint (variant 3);
    # 128 channels split over CTAs whose voxel-side gradients add
    # atomically; without the weight gradient the padding is skipped
    from ffdas_b200.tune import schedule
    g = torch.Generator().manual_seed(11 + C)
    x, src, dst, offs, w = _problem(8, B=2, C=C, S=7, N=140)
    V = dst.shape[:-1]
    n = 5
    idx = torch.randint(0, 7, (n, *V), generator=g).int()
    length = torch.randint(0, n + 1, V, generator=g)
    pad = torch.arange(n).reshape(n, 1, 1) >= length[None]
    ofs_s = (torch.rand((n, *V), generator=g) * 30 + 5).float()
    w_s = (torch.rand((n, *V), generator=g) + 0.2).float()
    w_s[pad] = 0.0
    need = [True, True, True, True, weights_grad]
    gpu = [t.to(DEV).requires_grad_(r) for t, r in zip((x, src, dst, ofs_s, w_s), need)]
    ref = [t.double().requires_grad_(r) for t, r in zip((x, src, dst, ofs_s, w_s), need)]
    gy = torch.randn((2, *V), generator=g)
    with schedule(dict(variant=3) if kernel == "gather" else None, DEV):
        ffdas_b200.das_sparse(*gpu, idx.to(DEV)).backward(gy.to(DEV))
        info = ffdas_b200.get_library_handle(DEV).last_kernel_info()
    das_ref(*ref, sparse_indices=idx).backward(gy.double())
    for name, a, b, r in zip(["x", "srcpos", "dstpos", "offsets", "weights"], gpu, ref, need):
        if not r:
            continue
        assert oracle.rel_l2(a.grad.cpu().numpy(), b.grad.numpy()) < 2e-4, name
    if kernel == "gather":
        assert info["variant"] == 3
        # 2 tiles of 4 x 64 voxels, one batch chunk of 2 items; 128 channels: 4 slices of 32
        assert info["grid"] == (8 if C == 128 else 2), info
    else:
        assert info["variant"] == 7
        # one 8 x 16 tile (7 x 9 voxels) per batch item; 128 channels: 4 slices of 32
        assert info["grid"] == (8 if C == 128 else 2), info


def _directivity(src, dst, frac=0.4):
    # elements facing +z with an acceptance threshold between two of the
    # problem's (voxel, element) cosines, so that no pair sits on the cone's
    # edge (there float32 and float64 could disagree on the mask)
    d = dst.reshape(-1, 1, 3).double() - src.reshape(1, -1, 3).double()
    cos = (d[..., 2] / d.norm(dim=-1)).flatten().sort().values
    # the widest gap among the cosines near the wanted fraction
    lo = int(frac * cos.numel())
    hi = min(cos.numel() - 1, lo + max(2, cos.numel() // 20))
    i = lo + int(torch.argmax(cos[lo + 1:hi + 1] - cos[lo:hi]))
    thr = float(0.5 * (cos[i] + cos[i + 1]))
    assert float(cos[i + 1] - cos[i]) > 1e-6
    sd = torch.zeros((src.shape[0], 4))
    sd[:, 2] = 1.0
    sd[:, 3] = thr
    return sd


@pytest.mark.parametrize("B", [1, 3])
def test_directivity_gradients_match_float64_reference(B):
    # element directivity masks taps as in the forward (the reference's
    # dir_check, das_alg1_kernels.cuh:72-76); the gradients follow the kept
    # taps (gather adjoint)
    cpu = list(_problem(5, B=B))
    sd = _directivity(cpu[1], cpu[2])
    gpu = [t.to(DEV).requires_grad_(True) for t in cpu]
    ref = [t.double().requires_grad_(True) for t in cpu]
    g = torch.randn((B, *cpu[2].shape[:-1]), generator=torch.Generator().manual_seed(6))
    out = das_autograd(*gpu, srcdir=sd.to(DEV))
    out.backward(g.to(DEV))
    out_ref = das_ref(*ref, srcdir=sd)
    out_ref.backward(g.double())
    masked = das_ref(*[t.detach().double() for t in cpu])
    assert oracle.rel_l2(out_ref.detach().numpy(), masked.numpy()) > 1e-2     # the mask removes taps
    assert oracle.rel_l2(out.detach().cpu().numpy(), out_ref.detach().numpy()) < 2e-5
    for name, a, b in zip(["x", "srcpos", "dstpos", "offsets", "weights"], gpu, ref):
        err = oracle.rel_l2(a.grad.cpu().numpy(), b.grad.numpy())
        assert err < 2e-4, (name, err)


def test_directivity_sparse_gradients_match_float64_reference():
    # das_sparse with directivity: the sorted-list adjoint applies the mask
    cpu = list(_problem(7, B=1, S=6))
    sd = _directivity(cpu[1], cpu[2], 0.5)
    g0 = torch.Generator().manual_seed(8)
    k = 3
    idx = torch.stack([torch.randperm(6, generator=g0)[:k] for _ in range(cpu[2][..., 0].numel())], -1)
    idx = idx.reshape(k, *cpu[2].shape[:-1]).int()
    offs = cpu[3][:k].clone()
    w = cpu[4][:k].clone()
    args = [cpu[0], cpu[1], cpu[2], offs, w]
    gpu = [t.to(DEV).requires_grad_(True) for t in args]
    ref = [t.double().requires_grad_(True) for t in args]
    g = torch.randn((1, *cpu[2].shape[:-1]), generator=torch.Generator().manual_seed(9))
    out = ffdas_b200.das_sparse(*gpu, idx.to(DEV), srcdir=sd.to(DEV))
    out.backward(g.to(DEV))
    out_ref = das_ref(*ref, sparse_indices=idx, srcdir=sd)
    out_ref.backward(g.double())
    assert oracle.rel_l2(out.detach().cpu().numpy(), out_ref.detach().numpy()) < 2e-5
    for name, a, b in zip(["x", "srcpos", "dstpos", "offsets", "weights"], gpu, ref):
        err = oracle.rel_l2(a.grad.cpu().numpy(), b.grad.numpy())
        assert err < 2e-4, (name, err)


@pytest.mark.parametrize("sparse, B, wavenum, C", [(False, 1, 0.0, 6), (False, 2, 0.07, 6), (True, 1, 0.05, 6),
                                                  (False, 2, 0.07, 64), (True, 1, 0.05, 64)])
def test_complex_gradients_match_float64_reference(sparse, B, wavenum, C):
    # complex IQ data with the phase rotation: the gradients of x (conj(A) g
    # split over the two taps), weights, delays (through the phase and the
    # slope) and both position sets against complex autograd of the float64
    # statement; with directivity for das_sparse; 64 channels run the
    # channel-sliced grid (slices add the voxel-side gradients)
    cpu = list(_problem(11, B=B, S=4, C=C))
    g0 = torch.Generator().manual_seed(12)
    cpu[0] = torch.complex(cpu[0], torch.randn(cpu[0].shape, generator=g0))
    idx = None
    if sparse:
        k = 3
        V = cpu[2][..., 0].numel()
        idx = torch.stack([torch.randperm(4, generator=g0)[:k] for _ in range(V)], -1)
        idx = idx.reshape(k, *cpu[2].shape[:-1]).int()
        cpu[3], cpu[4] = cpu[3][:k].clone(), cpu[4][:k].clone()
    sd = _directivity(cpu[1], cpu[2], 0.3) if sparse else None
    gpu = [t.to(DEV).requires_grad_(True) for t in cpu]
    ref = [(t.to(torch.complex128) if t.is_complex() else t.double()).requires_grad_(True) for t in cpu]
    g = torch.complex(torch.randn((B, *cpu[2].shape[:-1]), generator=g0),
                      torch.randn((B, *cpu[2].shape[:-1]), generator=g0))
    out = das_autograd(*gpu, idx.to(DEV) if sparse else None, srcdir=None if sd is None else sd.to(DEV),
                       wavenum=wavenum)
    out.backward(g.to(DEV))
    out_ref = das_ref(*ref, sparse_indices=idx, srcdir=sd, wavenum=wavenum)
    out_ref.backward(g.to(torch.complex128))
    assert oracle.rel_l2(out.detach().cpu().numpy(), out_ref.detach().numpy()) < 2e-5
    for name, a, b in zip(["x", "srcpos", "dstpos", "offsets", "weights"], gpu, ref):
        err = oracle.rel_l2(a.grad.cpu().numpy(), b.grad.numpy())
        assert err < 2e-4, (name, err)


def test_complex128_has_no_backward():
    cpu = list(_problem(13, B=1))
    x = torch.complex(cpu[0], cpu[0]).to(torch.complex128).to(DEV).requires_grad_(True)
    out = das_autograd(x, *[t.to(DEV) for t in cpu[1:]])
    with pytest.raises(NotImplementedError):
        out.abs().sum().backward()


def test_central_finite_differences_fp64():
    x, src, dst, offs, w = _problem(6, B=2)
    loss_ref = lambda o, ww: -(das_ref(x.double(), src.double(), dst.double(), o, ww) ** 4).sum()  # noqa: E731
    og = offs.to(DEV).requires_grad_(True)
    wg = w.to(DEV).requires_grad_(True)
    img = das_autograd(x.to(DEV), src.to(DEV), dst.to(DEV), og, wg)
    (-(img.double() ** 4).sum()).backward()
    rng = np.random.default_rng(7)
    h = 1e-4
    flat = offs.numel()
    picks = rng.choice(flat, 64, replace=False)
    checked = 0
    for var, grad in ((offs, og.grad), (w, wg.grad)):
        for i in picks[:32]:
            base = var.double().clone().reshape(-1)
            # skip delays whose perturbation crosses a sample boundary
            if var is offs:
                r = torch.sqrt(((dst.reshape(-1, 3)[i % dst[..., 0].numel()].double() - src.double()) ** 2).sum(-1))
                frac = (float(base[i]) + r) % 1.0
                if bool(((frac < 10 * h) | (frac > 1 - 10 * h)).any()):
                    continue
            p, m = base.clone(), base.clone()
            p[i] += h
            m[i] -= h
            args = [p.reshape(var.shape), w.double()] if var is offs else [offs.double(), p.reshape(var.shape)]
            argm = [m.reshape(var.shape), w.double()] if var is offs else [offs.double(), m.reshape(var.shape)]
            fd = float(loss_ref(*args) - loss_ref(*argm)) / (2 * h)
            an = float(grad.reshape(-1)[i])
            assert abs(fd - an) <= 2e-3 * max(abs(fd), 1e-3 * float(abs(grad).max())), (i, fd, an)
            checked += 1
    assert checked >= 40


def test_bf16_and_fp16_inputs_get_gradients():
    x, src, dst, offs, w = _problem(8, B=2)
    for dt in (torch.float16, torch.bfloat16):
        xg = x.to(DEV, dt).requires_grad_(True)
        wg = w.to(DEV).requires_grad_(True)
        out = das_autograd(xg, src.to(DEV), dst.to(DEV), offs.to(DEV), wg)
        out.sum().backward()
        assert xg.grad.dtype == dt and torch.isfinite(xg.grad.float()).all()
        ref_w = das_ref(x.to(dt).double(), src.double(), dst.double(), offs.double(),
                        w.double().requires_grad_(True))
        assert torch.isfinite(wg.grad).all()


def test_autofocus_recovers_sound_speed_scale():
    """50 Adam steps on alpha (init 1.0, true 1.03), loss = -sum |image|^4 with
    |image| the magnitude of the beamformed analytic signal (das is linear, so
    the real and imaginary parts are beamformed as two batch halves)."""
    wl = W.autofocus(device=DEV, scale=0.5, batch=2)
    xa = W.analytic_signal(wl["x"].double())
    xc = torch.cat([xa.real, xa.imag], 0).float().contiguous()
    B = wl["x"].shape[0]
    srcpos, dstpos, base, w = wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"]
    alpha = torch.tensor(1.0, device=DEV, requires_grad=True)
    opt = torch.optim.Adam([alpha], lr=4e-3)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, T_max=50)
    ref = None
    for _ in range(50):
        opt.zero_grad()
        img = ffdas_b200.das(xc, srcpos * alpha, dstpos * alpha, base * alpha, w)
        e2 = img[:B] ** 2 + img[B:] ** 2
        s = (e2 ** 2).sum()
        ref = float(s) if ref is None else ref
        (-s / ref).backward()
        opt.step()
        sched.step()
    assert abs(float(alpha) - wl["alpha_true"]) < 0.004, float(alpha)


def test_staged_and_gather_adjoints_agree():
    # dense problems take the staged adjoint unless the schedule asks for the
    # gather adjoint (variant 3); a forward schedule choice does not switch it
    from ffdas_b200.tune import schedule
    x, src, dst, offs, w = (t.to(DEV) for t in _problem(9, B=3, nz=40, nx=36))
    h = ffdas_b200.get_library_handle(DEV)
    grads, kinds = [], []
    for cfg in (None, dict(variant=1, batch_tile=2), dict(variant=2, copy_engine=2), dict(variant=3)):
        leaves = [t.clone().requires_grad_(True) for t in (x, src, dst, offs, w)]
        with schedule(cfg, DEV):
            das_autograd(*leaves).square().sum().backward()
            kinds.append(h.last_kernel_info()["variant"])
        grads.append([t.grad for t in leaves])
    assert kinds == [4, 4, 4, 3]
    for staged in grads[:3]:
        for a, b in zip(staged, grads[3]):
            assert oracle.rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-5


@pytest.mark.parametrize("B", [1, 3])
def test_channel_sliced_adjoint(B):
    # many CTAs per SM asked for: each voxel tile's 100 channels are split over
    # two CTAs (64 + 36 channels) that add into the voxel-side gradients.  The
    # sliced staged adjoint must agree with the gather adjoint (same per-tap
    # arithmetic) to 1e-5; x and weight gradients, which are continuous in the
    # delays, also match the float64 reference.  (Delay-driven gradients are
    # piecewise in the delay: on 4e5 taps a few lie within an fp32 rounding of
    # a sample boundary, so they are not compared with float64 here.)
    from ffdas_b200.tune import schedule
    cpu = _problem(11, B=B, C=100, nz=40, nx=36)
    g = torch.randn((B, *cpu[2].shape[:-1]), generator=torch.Generator().manual_seed(12))
    ref = [t.double().requires_grad_(True) for t in cpu]
    das_ref(*ref).backward(g.double())
    h = ffdas_b200.get_library_handle(DEV)
    grads = []
    for cfg in (dict(variant=2, tile_x=8, tile_y=32, min_blocks=32), dict(variant=3)):
        gpu = [t.to(DEV).requires_grad_(True) for t in cpu]
        with schedule(cfg, DEV):
            das_autograd(*gpu).backward(g.to(DEV))
            info = h.last_kernel_info()
        grads.append([t.grad for t in gpu])
        if cfg["variant"] == 2:
            bt = min(4, 1 << (B.bit_length() - 1))
            tiles = ((36 + 7) // 8) * ((40 + 31) // 32) * ((B + bt - 1) // bt)
            assert info["variant"] == 4 and info["grid"] == tiles * 2, info
    for name, a, b in zip(["x", "srcpos", "dstpos", "offsets", "weights"], *grads):
        assert oracle.rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-5, name
    for i in (0, 4):
        assert oracle.rel_l2(grads[0][i].cpu().numpy(), ref[i].grad.numpy()) < 2e-4


def test_backward_reads_the_forward_pair_rows():
    # the autograd forward builds its pair rows into a buffer kept for the
    # backward (ffdas_set_pair_buffer); the backward then launches only the
    # adjoint kernel, and its gradients match those of a backward that builds
    # the rows again
    from ffdas_b200 import _lib
    from ffdas_b200._lib import DataType
    wl = W.autofocus(device=DEV, scale=0.25)
    h = ffdas_b200.get_library_handle(DEV)
    leaves = [t.clone().requires_grad_(True) for t in (wl["x"], wl["offsets"], wl["weights"])]
    out = ffdas_b200.das(leaves[0], wl["srcpos"], wl["dstpos"], leaves[1], leaves[2])
    out.square().sum().backward()
    assert h.last_kernel_info()["kernels"] == 1
    grads = [t.grad.clone() for t in leaves]
    # the same backward through the C-ABI without the buffer: ingest + adjoint
    x = wl["x"]
    gout = 2 * out.detach()
    gx = torch.zeros_like(x)
    go = torch.empty_like(wl["offsets"])
    gw = torch.empty_like(wl["weights"])
    xd = _lib.TensorDesc(list(x.shape), list(x.stride()), DataType.R_32F)
    gd = _lib.TensorDesc(list(gout.shape), None, DataType.R_32F)
    h.set_stream(torch.cuda.current_stream().cuda_stream)
    _lib.check(_lib.load().ffdas_das_backward(h.h, wl["srcpos"].data_ptr(), None, 0.0, xd.desc, x.data_ptr(),
                                              wl["dstpos"].data_ptr(), wl["offsets"].data_ptr(),
                                              wl["weights"].data_ptr(), 0, None, gd.desc, gout.data_ptr(),
                                              gx.data_ptr(), go.data_ptr(), gw.data_ptr(), None, None))
    assert h.last_kernel_info()["kernels"] == 2
    torch.cuda.synchronize()
    # equal up to the order of the float atomics that add the tiles' gradients
    for a, b in zip(grads, (gx, go, gw)):
        assert oracle.rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-6
