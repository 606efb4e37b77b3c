"""GPU tests of the surrogate's tensor-core kernels.

* lcb_mlp_gemm (tcgen05 + TMEM + TMA) against a torch FP32 matmul of the same
  BF16 operands, every epilogue mode, ragged and multi-stage shapes;
* forward/backward of the whole network against the FP64 CPU oracle
  (oracle/mlp_oracle.py), which rounds to BF16 at the same points;
* a short training run lowers the loss.

Tolerances are written beside each check.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _gemm(lcb, mode, A, B, bias=None, aux=None):
    M, K = A.shape
    N = B.shape[0]
    dev = A.device
    if mode in (0, 2):
        out = torch.empty(M, N, device=dev, dtype=torch.float32)
    else:
        out = torch.empty(M, N, device=dev, dtype=torch.bfloat16)
    out2 = torch.empty(M, N, device=dev, dtype=torch.float32) if mode == 1 else None
    err = torch.zeros(1, device=dev, dtype=torch.int32)
    L = lcb._capi.load()
    lcb._capi.check_mlp(L.lcb_mlp_gemm(mode, M, N, K, _ptr(A), _ptr(B), _ptr(bias), _ptr(aux), _ptr(out), _ptr(out2),
                                       _ptr(err), None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return out, out2


@pytest.mark.parametrize("M,N,K", [(300, 136, 200), (4096, 512, 512), (128, 8, 1024), (77, 256, 8)])
def test_gemm_matches_torch(lcb, M, N, K):
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    aux = torch.randn(M, N, device="cuda", generator=g)
    ref = A.float() @ B.float().T
    # bound on accumulation-order differences: FP32 epsilon x sum of |terms|
    bound = 4e-6 * (A.float().abs() @ B.float().abs().T) + 1e-6
    out, _ = _gemm(lcb, 0, A, B)
    assert bool(((out - ref).abs() <= bound).all())
    out, _ = _gemm(lcb, 2, A, B, bias=bias)
    assert bool(((out - (ref + bias)).abs() <= bound).all())
    y, z = _gemm(lcb, 1, A, B, bias=bias)
    assert bool(((z - (ref + bias)).abs() <= bound).all())
    gelu = torch.nn.functional.gelu(z)  # exact erf form; compare after BF16 rounding (one BF16 ulp = 2^-8 relative)
    assert bool(((y.float() - gelu).abs() <= 2 ** -8 * gelu.abs() + 1e-6).all())
    d, _ = _gemm(lcb, 3, A, B, aux=aux)
    zz = aux.clone().requires_grad_(True)
    torch.nn.functional.gelu(zz).sum().backward()
    dref = ref * zz.grad
    assert bool(((d.float() - dref).abs() <= 2 ** -8 * dref.abs() + bound * zz.grad.abs() + 1e-6).all())


SHAPE = dict(n_in=5, width=512, n_hidden=4, n_out=256)


def _net(lcb, seed=11, max_batch=1024):
    L = lcb._capi.load()
    h = C.c_void_p()
    lcb._capi.check_mlp(L.lcb_mlp_create(0, SHAPE["n_in"], SHAPE["width"], SHAPE["n_hidden"], SHAPE["n_out"],
                                         max_batch, seed, C.byref(h)))
    n = C.c_int64()
    lcb._capi.check_mlp(L.lcb_mlp_num_params(h, C.byref(n)))
    return L, h, n.value


def test_backward_matches_cpu_oracle(lcb):
    from oracle import mlp_oracle as MO

    L, h, n = _net(lcb)
    try:
        assert n == 5 * 512 + 512 + 3 * (512 * 512 + 512) + 512 * 256 + 256
        rng = np.random.default_rng(3)
        B = 192
        x = rng.uniform(-1, 1, (B, 5)).astype(np.float32)
        t = rng.normal(0, 1, (B, 256)).astype(np.float32)
        params = np.empty(n, np.float32)
        lcb._capi.check_mlp(L.lcb_mlp_get_params(h, params.ctypes.data, n))
        xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
        y = torch.empty(B, 256, device="cuda")
        torch.cuda.synchronize()  # the network works on its own stream
        lcb._capi.check_mlp(L.lcb_mlp_forward(h, _ptr(xd), B, _ptr(y)))
        lcb._capi.check_mlp(L.lcb_mlp_sync(h))
        y = y.cpu().numpy()
        lcb._capi.check_mlp(L.lcb_mlp_backward(h, _ptr(xd), _ptr(td), B))
        grads = np.empty(n, np.float32)
        lcb._capi.check_mlp(L.lcb_mlp_get_grads(h, grads.ctypes.data, n))
        loss = C.c_double()
        lcb._capi.check_mlp(L.lcb_mlp_take_loss(h, C.byref(loss)))
        ref_loss, ref_grads, ref_pred = MO.loss_and_grads(params.astype(np.float64), x, t, **SHAPE)
        # forward: FP32 accumulation vs FP64 on identical BF16 operands
        assert np.max(np.abs(y - ref_pred)) <= 1e-3 * np.max(np.abs(ref_pred)) + 1e-4
        assert abs(loss.value - ref_loss) <= 1e-3 * ref_loss
        # gradients, layer by layer: norm-relative error below 1e-2 (BF16 rounding of the
        # inter-layer gradients can flip by one ulp where the two sums straddle a tie)
        k = 0
        shapes = [(512, 5)] + [(512, 512)] * 3 + [(256, 512)]
        for (o, i) in shapes:
            for size in (o * i, o):
                g, r = grads[k:k + size], ref_grads[k:k + size]
                assert np.linalg.norm(g - r) <= 1e-2 * np.linalg.norm(r) + 1e-12, (k, size)
                k += size
    finally:
        L.lcb_mlp_destroy(h)


def test_training_lowers_the_loss(lcb):
    L, h, n = _net(lcb, seed=5, max_batch=4096)
    try:
        g = torch.Generator(device="cuda").manual_seed(0)
        x = torch.rand(4096, 5, device="cuda", generator=g) * 2 - 1
        w = torch.randn(5, 256, device="cuda", generator=g)
        t = torch.sin(x @ w)  # smooth target curves
        torch.cuda.synchronize()  # the network works on its own stream
        losses = []
        for step in range(300):
            lcb._capi.check_mlp(L.lcb_mlp_train_step(h, _ptr(x), _ptr(t), 4096, 1e-3, 0.9, 0.999, 1e-8, 0.0))
            if step % 50 == 49:
                v = C.c_double()
                lcb._capi.check_mlp(L.lcb_mlp_take_loss(h, C.byref(v)))
                losses.append(v.value / 50)
        assert losses[-1] < 0.1 * losses[0], losses
    finally:
        L.lcb_mlp_destroy(h)


def test_data_parallel_path_matches_single_process(lcb):
    """Surrogate.fit through its data-parallel path (backward, all-reduce of
    lcb_mlp_grads_device on the network's stream, lcb_mlp_adam_step) in a
    one-rank NCCL group: the kernels are deterministic and the reduction is
    the identity, so the weights equal the default path's bit for bit."""
    import importlib
    import socket
    from datetime import timedelta

    import torch.distributed as dist

    S = importlib.import_module("lcurve-rs_b200.surrogate")
    rng = np.random.default_rng(4)
    theta = S.sample_prior(4096, seed=5)
    phase = np.linspace(0.0, 1.0, 256)
    flux = 1.0 + 0.2 * np.sin(2 * np.pi * phase[None, :] + 3 * theta[:, :1]) * theta[:, 2:3] / 0.03
    flux *= 1.0 + 0.01 * rng.random(flux.shape)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=120), device_id=torch.device("cuda", 0))
    try:
        out = []
        for group in (None, dist.group.WORLD):
            sur = S.Surrogate(seed=3, max_batch=1024)
            losses = sur.fit(theta, flux, epochs=3, batch=1024, group=group)
            n = C.c_int64()
            lcb._capi.check_mlp(sur.L.lcb_mlp_num_params(sur._h, C.byref(n)))
            p = np.empty(n.value, np.float32)
            lcb._capi.check_mlp(sur.L.lcb_mlp_get_params(sur._h, p.ctypes.data, n.value))
            out.append((p, losses))
        assert np.array_equal(out[0][0], out[1][0])
        assert np.allclose(out[0][1], out[1][1], rtol=1e-9)  # the loss sum uses FP64 atomics
        assert out[0][1][-1] < out[0][1][0]
    finally:
        dist.destroy_process_group()


def test_checkpoint_resumes_training_exactly(lcb, tmp_path):
    """Surrogate.save after some training, then Surrogate.load into a fresh
    network and the same further training: the weights equal those of the
    uninterrupted run bit for bit (parameters, Adam moments and step count
    are restored; the kernels are deterministic)."""
    import importlib
    S = importlib.import_module("lcurve-rs_b200.surrogate")
    rng = np.random.default_rng(8)
    theta = S.sample_prior(2048, seed=6)
    phase = np.linspace(0.0, 1.0, 256)
    flux = 1.0 + 0.2 * np.cos(2 * np.pi * phase[None, :] + 2 * theta[:, 1:2] / 90.0) * theta[:, 2:3] / 0.03
    flux *= 1.0 + 0.01 * rng.random(flux.shape)

    def params(sur):
        n = C.c_int64()
        lcb._capi.check_mlp(sur.L.lcb_mlp_num_params(sur._h, C.byref(n)))
        p = np.empty(n.value, np.float32)
        lcb._capi.check_mlp(sur.L.lcb_mlp_get_params(sur._h, p.ctypes.data, n.value))
        return p

    a = S.Surrogate(seed=11, max_batch=1024)
    a.fit(theta, flux, epochs=2, batch=1024)
    a.save(tmp_path / "sur.npz")
    a.fit(theta, flux, epochs=2, batch=1024, renormalize=False)
    b = S.Surrogate.load(tmp_path / "sur.npz")
    b.fit(theta, flux, epochs=2, batch=1024, renormalize=False)
    assert np.array_equal(params(a), params(b))
    assert np.array_equal(a.predict(theta[:64]), b.predict(theta[:64]))
