"""Learned warm start of the CG solve that replaces the PETSc path (no counterpart in the reference, whose solve
starts from zero; SOLVE_POTENTIAL_WITH_PETSC, src/pic2d_ElectricFieldCalc_PETSc.F90:7-355).

A 4-level convolutional encoder-decoder (channels 32-64-128-256, 3x3 kernels, 4x4 average pooling so that the
bottleneck sees the whole domain, nearest upsampling, skip concatenation, ReLU, BF16 weights and activations with FP32 accumulation; LAYERS below) maps the
residual r0 = b - A phi_prev of the previous potential against the new charge density, divided by its RMS s, and the
Dirichlet mask to the update (phi - phi_prev) / s = K o0 + o1 through two FP32 heads, K = L^2 / (2 pi^2): o0 carries
the smooth part (the inverse Laplacian grows like L^2 on the longest wavelengths) and o1 the grid-scale part, so both
stay O(1) inside the BF16 network. Since A phi = b, r0 = A (phi - phi_prev): a training sample is one potential update
of a plain run.

Training runs on the device kernels of libedipic_b200.so (edp_nn_*) behind torch.autograd.Function wrappers; torch
holds the tensors and chains the backward pass, the loss is torch arithmetic, and the Adam step is the library's.
The parameters travel as one FP32 vector in the order the C ABI (edp_warmstart_load) reads.
"""
import ctypes as C
import math

import numpy as np

from . import library

LAYERS = [(32, 32), (32, 32), (32, 64), (64, 64), (64, 128), (128, 128), (128, 256), (256, 256), (384, 128),
          (128, 128), (192, 64), (64, 64), (96, 32), (32, 32)]
HEAD_C = 32
IN_C = 32   # input channels: residual / s, Dirichlet mask, zeros
POOL = 4    # pooling / upsampling factor per level


N_HEADS = 2   # smooth (scaled by K) and grid-scale outputs


def param_layout():
    """[(w_offset, b_offset, cin, cout)] per convolution, [(wh_offset, bh_offset)] per head, total count."""
    out, off = [], 0
    for ci, co in LAYERS:
        out.append((off, off + 9 * ci * co, ci, co))
        off += 9 * ci * co + co
    heads = []
    for _ in range(N_HEADS):
        heads.append((off, off + 9 * HEAD_C))
        off += 9 * HEAD_C + 1
    return out, heads, off


def n_params():
    return param_layout()[2]


def init_params(seed=0):
    """He-normal convolution weights and zero biases; the K-scaled head starts at zero (K is ~10^4 on a 512-cell
    grid, so a random start would swamp the first updates), the grid-scale head small."""
    rng = np.random.default_rng(seed)
    convs, heads, n = param_layout()
    theta = np.zeros(n, dtype=np.float32)
    for (wo, bo, ci, co) in convs:
        theta[wo:bo] = rng.normal(0.0, math.sqrt(2.0 / (9 * ci)), 9 * ci * co)
    wh, bh = heads[1]
    theta[wh:bh] = rng.normal(0.0, 0.1 * math.sqrt(1.0 / (9 * HEAD_C)), 9 * HEAD_C)
    return theta


def padded(n):
    """grid size of the network image: three poolings by POOL"""
    m = POOL ** 3
    return (n + m - 1) // m * m


def k_factor(ncx, ncy):
    L = float(max(ncx, ncy))
    return L * L / (2.0 * math.pi * math.pi)


def _torch():
    import torch
    return torch


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} returned {rc}")


def _fns():
    """The autograd Functions over the library kernels (built lazily: torch is imported only when training)."""
    torch = _torch()
    lib = library()

    def stream():
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    class Conv3x3(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x1, x2, w32, b32, wbf, cout, relu):
            n, h, w, c1 = x1.shape
            c2 = x2.shape[-1] if x2 is not None else 0
            y = torch.empty((n, h, w, cout), device=x1.device, dtype=torch.bfloat16)
            _check(lib.edp_nn_conv3x3_fwd(n, h, w, _ptr(x1), c1, _ptr(x2), c2, _ptr(wbf), _ptr(b32), cout, relu,
                                          _ptr(y), stream()), "conv3x3_fwd")
            ctx.save_for_backward(x1, x2, wbf, y)
            ctx.dims = (n, h, w, c1, c2, cout, relu)
            return y

        @staticmethod
        def backward(ctx, dy):
            x1, x2, wbf, y = ctx.saved_tensors
            n, h, w, c1, c2, cout, relu = ctx.dims
            dy = dy.contiguous()
            if relu:
                dz = torch.empty_like(dy)
                _check(lib.edp_nn_relu_bwd(n * h * w, cout, _ptr(dy), cout, 0, None, _ptr(y), _ptr(dz), stream()),
                       "relu_bwd")
            else:
                dz = dy
            cin = c1 + c2
            dw = torch.zeros((cout, 9, cin), device=dy.device, dtype=torch.float32)
            db = torch.zeros(cout, device=dy.device, dtype=torch.float32)
            _check(lib.edp_nn_conv3x3_wgrad(n, h, w, _ptr(x1), c1, _ptr(x2), c2, _ptr(dz), cout, _ptr(dw), _ptr(db),
                                            stream()), "conv3x3_wgrad")
            dx1 = dx2 = None
            if ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
                wt = torch.empty((cin, 9, cout), device=dy.device, dtype=torch.bfloat16)
                _check(lib.edp_nn_flip_transpose(_ptr(wbf), cout, cin, _ptr(wt), stream()), "flip_transpose")
                dx = torch.empty((n, h, w, cin), device=dy.device, dtype=torch.bfloat16)
                _check(lib.edp_nn_conv3x3_fwd(n, h, w, _ptr(dz), cout, None, 0, _ptr(wt), None, cin, 0, _ptr(dx),
                                              stream()), "conv3x3_dgrad")
                dx1 = dx[..., :c1].contiguous()
                dx2 = dx[..., c1:].contiguous() if c2 else None
            return dx1, dx2, dw.view(-1), db, None, None, None

    class Pool(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x):
            n, h, w, c = x.shape
            y = torch.empty((n, h // POOL, w // POOL, c), device=x.device, dtype=torch.bfloat16)
            _check(lib.edp_nn_pool(n, h, w, c, POOL, _ptr(x), _ptr(y), stream()), "pool")
            ctx.dims = (n, h, w, c)
            return y

        @staticmethod
        def backward(ctx, dy):
            n, h, w, c = ctx.dims
            dx = torch.empty((n, h, w, c), device=dy.device, dtype=torch.bfloat16)
            _check(lib.edp_nn_pool_bwd(n, h, w, c, POOL, _ptr(dy.contiguous()), _ptr(dx), 0, stream()), "pool_bwd")
            return dx

    class Up(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x):
            n, h, w, c = x.shape
            y = torch.empty((n, POOL * h, POOL * w, c), device=x.device, dtype=torch.bfloat16)
            _check(lib.edp_nn_upsample(n, POOL * h, POOL * w, c, POOL, _ptr(x), _ptr(y), stream()), "upsample")
            ctx.dims = (n, POOL * h, POOL * w, c)
            return y

        @staticmethod
        def backward(ctx, dy):
            n, h, w, c = ctx.dims
            dx = torch.empty((n, h // POOL, w // POOL, c), device=dy.device, dtype=torch.bfloat16)
            _check(lib.edp_nn_upsample_bwd(n, h, w, c, c, POOL, _ptr(dy.contiguous()), _ptr(dx), stream()),
                   "upsample_bwd")
            return dx

    class Head(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x, wh, bh):
            n, h, w, c = x.shape
            out = torch.empty((n, h, w), device=x.device, dtype=torch.float32)
            _check(lib.edp_nn_head_fwd(n, h, w, c, _ptr(x), _ptr(wh), _ptr(bh), _ptr(out), stream()), "head_fwd")
            ctx.save_for_backward(x, wh)
            ctx.dims = (n, h, w, c)
            return out

        @staticmethod
        def backward(ctx, dout):
            x, wh = ctx.saved_tensors
            n, h, w, c = ctx.dims
            dx = torch.empty_like(x)
            dwh = torch.zeros_like(wh)
            dbh = torch.zeros(1, device=x.device, dtype=torch.float32)
            _check(lib.edp_nn_head_bwd(n, h, w, c, _ptr(x), _ptr(wh), _ptr(dout.contiguous()), _ptr(dx), _ptr(dwh),
                                       _ptr(dbh), stream()), "head_bwd")
            return dx, dwh, dbh

    return Conv3x3, Pool, Up, Head


class WarmStartNet:
    """The network on the current CUDA device: FP32 master parameters (one leaf tensor), their BF16 copy, Adam
    moments."""

    def __init__(self, theta=None, seed=0):
        torch = _torch()
        if theta is None:
            theta = init_params(seed)
        self.theta = torch.tensor(np.asarray(theta, dtype=np.float32), device="cuda").requires_grad_(True)
        self.theta_bf = self.theta.detach().to(torch.bfloat16)
        self.m = torch.zeros_like(self.theta.detach())
        self.v = torch.zeros_like(self.theta.detach())
        self.steps = 0
        self.convs, self.heads, _ = param_layout()
        self.Conv3x3, self.Pool, self.Up, self.Head = _fns()

    def _conv(self, l, x1, x2=None, relu=1):
        wo, bo, ci, co = self.convs[l]
        w32 = self.theta[wo:bo]
        b32 = self.theta[bo:bo + co]
        wbf = self.theta_bf[wo:bo]
        return self.Conv3x3.apply(x1, x2, w32, b32, wbf, co, relu)

    def forward(self, x):
        """x: [images, H, W, 32] BF16 (H, W multiples of 64) -> (o0, o1), each [images, H, W] FP32."""
        P, U = self.Pool.apply, self.Up.apply
        s0 = self._conv(1, self._conv(0, x))
        s1 = self._conv(3, self._conv(2, P(s0)))
        s2 = self._conv(5, self._conv(4, P(s1)))
        bb = self._conv(7, self._conv(6, P(s2)))
        d2 = self._conv(9, self._conv(8, U(bb), s2))
        d1 = self._conv(11, self._conv(10, U(d2), s1))
        d0 = self._conv(13, self._conv(12, U(d1), s0))
        return tuple(self.Head.apply(d0, self.theta[wh:bh], self.theta[bh:bh + 1]) for (wh, bh) in self.heads)

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        torch = _torch()
        self.steps += 1
        lib = library()
        _check(lib.edp_nn_adam(_ptr(self.theta), _ptr(self.theta.grad), _ptr(self.m), _ptr(self.v),
                               self.theta.numel(), lr, beta1, beta2, eps, self.steps, _ptr(self.theta_bf),
                               C.c_void_p(torch.cuda.current_stream().cuda_stream)), "adam")
        self.theta.grad = None

    def blob(self):
        return self.theta.detach().cpu().numpy().astype(np.float32)


# ------------------------------------------------------------------------------------------ samples and loss
def stencil(t, unk):
    """A t on the unknown nodes (4 t - neighbours; t is zero off the unknowns), batched [N, H, W] FP32."""
    torch = _torch()
    z = t * unk
    p = torch.nn.functional.pad(z, (1, 1, 1, 1))
    a = 4.0 * z - p[:, 1:-1, :-2] - p[:, 1:-1, 2:] - p[:, :-2, 1:-1] - p[:, 2:, 1:-1]
    return a * unk


def make_batch(dphi, unk):
    """Network input, normalised target and masks from potential updates dphi [N, H, W] (zero off the unknowns) and
    unknown-node masks unk [N, H, W] (1.0 / 0.0), FP32 on the device."""
    torch = _torch()
    r0 = stencil(dphi, unk)
    n_unk = unk.sum(dim=(1, 2)).clamp_min(1.0)
    s = torch.sqrt((r0 * r0).sum(dim=(1, 2)) / n_unk).clamp_min(1e-30)
    rhat = r0 / s[:, None, None]
    x = torch.zeros(tuple(dphi.shape) + (IN_C,), device=dphi.device, dtype=torch.bfloat16)
    x[..., 0] = rhat.to(torch.bfloat16)
    x[..., 1] = (1.0 - unk).to(torch.bfloat16)
    return x, rhat, dphi / s[:, None, None]


def losses(out, rhat, t, unk, K):
    """Per-sample relative residual |r0 - A u|^2 / |r0|^2 and relative energy-norm error |t - u|_A^2 / |t|_A^2 of
    the normalised update u = K o0 + o1, as the CG start phi_prev + s u would see them."""
    u = (K * out[0].double() + out[1].double()) * unk
    r1 = rhat - stencil(u, unk)
    lr = (r1 * r1).sum(dim=(1, 2)) / (rhat * rhat).sum(dim=(1, 2)).clamp_min(1e-30)
    e = (t - u) * unk
    le = (e * stencil(e, unk)).sum(dim=(1, 2)) / (t * rhat).sum(dim=(1, 2)).clamp_min(1e-30)
    return lr, le


def train(net, dphi, unk, K, steps=500, batch=4, lr=1e-3, seed=0, log=None):
    """Adam on the summed relative residual and energy-norm losses over random minibatches of the samples."""
    torch = _torch()
    g = torch.Generator(device="cpu").manual_seed(seed)
    n = dphi.shape[0]
    hist = []
    for it in range(steps):
        idx = torch.randint(0, n, (min(batch, n),), generator=g).to(dphi.device)
        x, rhat, t = make_batch(dphi[idx], unk[idx])
        out = net.forward(x)
        lr_, le_ = losses(out, rhat, t, unk[idx], K)
        loss = (lr_ + le_).mean()
        loss.backward()
        net.adam_step(lr)
        if log is not None and (it % 50 == 0 or it == steps - 1):
            hist.append((it, float(lr_.mean()), float(le_.mean())))
            log(f"step {it}: residual {hist[-1][1]:.4f} energy {hist[-1][2]:.4f}")
    return hist


def generate_samples(deck_dirs, steps_per_deck, warmup=4, precision=None, rtol=1e-10, ppc=None):
    """Potential updates of plain runs: for every deck, the cycle is stepped with CG (multigrid preconditioner,
    previous-step warm start, tolerance rtol) and phi_n - phi_(n-1) is kept for every step after warmup.
    Returns (dphi [N, H, W] FP64, unk [N, H, W] FP64) on the device, padded for the network (FP64 keeps the residual
    A dphi of smooth updates free of cancellation)."""
    torch = _torch()
    from . import FIELD_PHI, PREC_MIXED, Simulation
    out_d, out_u = [], []
    for d in deck_dirs:
        with Simulation(d, precision=PREC_MIXED if precision is None else precision, sort_every=20) as sim:
            p = sim.params
            sim.distribute_particles(ppc or p.n_of_particles_cell)
            ny, nx = p.ncy + 1, p.ncx + 1
            H, W = padded(ny), padded(nx)
            unk = np.zeros((H, W), dtype=np.float64)
            unk[1:ny - 1, 1:nx - 1] = 1.0
            for o in range(p.n_inner):
                unk[p.inner_jbottom[o]:p.inner_jtop[o] + 1, p.inner_ileft[o]:p.inner_iright[o] + 1] = 0.0
            prev = None
            for k in range(warmup + steps_per_deck):
                sim.update_wall_potentials(k)
                sim.solve_potential_with_cg(rtol=rtol, max_it=100000)
                phi = sim.field(FIELD_PHI)
                if prev is not None and k >= warmup:
                    dp = np.zeros((H, W), dtype=np.float64)
                    dp[:ny, :nx] = (phi - prev) * unk[:ny, :nx]
                    out_d.append(dp)
                    out_u.append(unk)
                prev = phi
                sim.advance_electrons()
                sim.advance_ions()
                sim.perform_electron_neutral_collisions()
                sim.perform_resonant_charge_exchange()
                sim.end_ion_cycle()
    dphi = torch.tensor(np.stack(out_d), device="cuda")
    unk = torch.tensor(np.stack(out_u), device="cuda")
    return dphi, unk


# ------------------------------------------------------------------------------------------ cfg3 family
def cfg3_geometries(n, seed=0, ncx=512, ncy=512):
    """Object rectangles of the learned-warm-start training set: 64 x 32 cells centred at (256, 128) jittered by up to
    +-64 cells per axis, biased uniformly in [-200, 0] V (scaled to the grid when it is not 512 x 512)."""
    rng = np.random.default_rng(seed)
    sx, sy = ncx / 512.0, ncy / 512.0
    out = []
    for _ in range(n):
        cx = int(round((256 + rng.uniform(-64, 64)) * sx))
        cy = int(round((128 + rng.uniform(-64, 64)) * sy))
        hw, hh = max(1, int(round(32 * sx))), max(1, int(round(16 * sy)))
        out.append((cx - hw, cy - hh, cx + hw, cy + hh, float(rng.uniform(-200.0, 0.0))))
    return out


def save_blob(path, theta):
    """Convolution weights as BF16 bits (the device uses them as BF16), biases and head as FP32."""
    convs, _, n = param_layout()
    theta = np.asarray(theta, dtype=np.float32)
    wmask = np.zeros(n, dtype=bool)
    for (wo, bo, ci, co) in convs:
        wmask[wo:bo] = True
    bits = theta[wmask].view(np.uint32)
    bits = ((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16).astype(np.uint16)
    np.savez_compressed(path, w_bf16=bits, rest_f32=theta[~wmask], n=np.int64(n))


def load_blob(path):
    z = np.load(path)
    convs, _, n = param_layout()
    if int(z["n"]) != n:
        raise ValueError(f"{path}: {int(z['n'])} parameters, the network has {n}")
    wmask = np.zeros(n, dtype=bool)
    for (wo, bo, ci, co) in convs:
        wmask[wo:bo] = True
    theta = np.zeros(n, dtype=np.float32)
    theta[wmask] = (z["w_bf16"].astype(np.uint32) << 16).view(np.float32)
    theta[~wmask] = z["rest_f32"]
    return theta


# ------------------------------------------------------------------------------------------ layer timing
def time_layer(cin, cout, h, w, nimg, reps=10):
    """CUDA-event time (us) and TFLOP/s of one forward convolution of the network's kind on random data."""
    torch = _torch()
    lib = library()
    st = torch.cuda.current_stream()
    x = torch.randn(nimg, h, w, cin, device="cuda").to(torch.bfloat16)
    y = torch.empty(nimg, h, w, cout, device="cuda", dtype=torch.bfloat16)
    wt = (torch.randn(cout, 9, cin, device="cuda") * 0.05).to(torch.bfloat16)
    b = torch.zeros(cout, device="cuda")
    args = (nimg, h, w, _ptr(x), cin, None, 0, _ptr(wt), _ptr(b), cout, 1, _ptr(y), C.c_void_p(st.cuda_stream))
    for _ in range(3):
        _check(lib.edp_nn_conv3x3_fwd(*args), "conv3x3_fwd")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        lib.edp_nn_conv3x3_fwd(*args)
    e1.record(st)
    e1.synchronize()
    t = e0.elapsed_time(e1) / reps * 1e-3
    return t * 1e6, 2.0 * nimg * h * w * 9 * cin * cout / t / 1e12


def time_wgrad(cin, cout, h, w, nimg, reps=10):
    """CUDA-event time (us) and TFLOP/s of one weight gradient (with the bias gradient) of the network's kind."""
    torch = _torch()
    lib = library()
    st = torch.cuda.current_stream()
    x = torch.randn(nimg, h, w, cin, device="cuda").to(torch.bfloat16)
    dz = torch.randn(nimg, h, w, cout, device="cuda").to(torch.bfloat16)
    dw = torch.zeros(cout, 9, cin, device="cuda")
    db = torch.zeros(cout, device="cuda")
    args = (nimg, h, w, _ptr(x), cin, None, 0, _ptr(dz), cout, _ptr(dw), _ptr(db), C.c_void_p(st.cuda_stream))
    for _ in range(3):
        _check(lib.edp_nn_conv3x3_wgrad(*args), "conv3x3_wgrad")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        lib.edp_nn_conv3x3_wgrad(*args)
    e1.record(st)
    e1.synchronize()
    t = e0.elapsed_time(e1) / reps * 1e-3
    return t * 1e6, 2.0 * nimg * h * w * 9 * cin * cout / t / 1e12


if __name__ == "__main__":
    # python -m edipic_b200.warmstart CIN COUT H W IMAGES [KERNEL]: times one forward convolution layer; KERNEL selects
    # the forward kernel as edp_nn_conv_select does (0 automatic, 1 tile, 2 persistent halo).
    # python -m edipic_b200.warmstart wgrad CIN COUT H W IMAGES [KERNEL]: the weight gradient instead; KERNEL as
    # edp_nn_wgrad_select (0 tcgen05 with the taps in M, 1 mma.sync, 2 tcgen05 with the taps in N)
    import sys
    argv = sys.argv[1:]
    wgrad = bool(argv) and argv[0] == "wgrad"
    if wgrad:
        argv = argv[1:]
    a = [int(v) for v in argv[0:5]]
    if len(argv) > 5:
        sel = library().edp_nn_wgrad_select if wgrad else library().edp_nn_conv_select
        _check(sel(int(argv[5])), "kernel select")
    us, tf = (time_wgrad if wgrad else time_layer)(*a)
    kind = "wgrad" if wgrad else "fwd"
    print(f"{kind} {a[0]}->{a[1]} {a[4]}x{a[2]}x{a[3]}: {us:.1f} us, {tf:.1f} TFLOP/s")
