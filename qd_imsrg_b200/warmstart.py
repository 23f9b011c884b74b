"""Learned warm start of the Magnus flow.

A small per-entry network predicts the Magnus operator Omega at a flow
parameter s from features of each of Omega's entries (fph and Vpphh: the
only parts the White-generator flow fills).  It predicts each entry as a
multiple of the first-order generator, Omega_e(s) = eta0_e * r_e(s) with
eta0 = build_white(H_HF) (the flow's own first step direction), so that its
error on an entry scales with that entry; an absolute error on each of the
~10^6 entries would add up to a large change of Omega.  The plain flow then continues
from the prediction (qd_flow_warm_start) to the reference's convergence
criterion; if the predicted state is worse than the Hartree-Fock start
(|MBPT2| not below its s = 0 value), the prediction is rejected and the flow
restarts from Omega = 0.  The plain flow's own trajectories are the training
data.

Every numeric step runs in the library's kernels (features, gather/scatter,
network forward/backward, Adam); torch tensors serve only as device buffers.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import FullHam, Flow, Layout, build_white, hf_hamiltonian, mbpt2
from ._native import check, lib

NFEAT = 16
NPARAM = 70401
RATIO_CLAMP = 4.0  # training targets r = Omega / eta0 are clipped to [-4, 4]
ETA_FLOOR = 1e-10  # entries with |eta0| below this are not trained on (Omega ~ 0 there)


def _torch():
    import torch

    return torch


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def omega_count(P: Layout) -> int:
    n = C.c_int64()
    check(lib().qd_omega_count(P.h, C.byref(n)))
    return n.value


def omega_gather(G: FullHam, out) -> None:
    """out (float64 device tensor, omega_count entries) = Omega entries of G."""
    check(lib().qd_omega_gather(G.h, _ptr(out), out.numel()))


def omega_scatter(G: FullHam, vals, scale: float, escale=None) -> None:
    """G = 0 except its Omega entries = scale * vals (float32 device tensor),
    times escale (float64 device tensor) entry by entry if given."""
    check(lib().qd_omega_scatter(G.h, _ptr(vals), float(scale), _ptr(escale) if escale is not None else None,
                                 vals.numel()))


def omega_features(H: FullHam, hw: float, s: float, out) -> None:
    """out (float32 device tensor [n, 16]) = features of every Omega entry."""
    check(lib().qd_omega_features(H.h, float(hw), float(s), _ptr(out), out.shape[0]))


class MLP:
    """The per-entry network (16 -> 256 -> 256 -> 1) on one device."""

    def __init__(self, device: int = 0, seed: int = 1):
        self.h = C.c_void_p()
        check(lib().qd_mlp_create(int(device), C.c_uint64(seed), C.byref(self.h)))
        self.device = device

    def params(self) -> np.ndarray:
        p = np.empty(NPARAM, np.float32)
        check(lib().qd_mlp_get_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), NPARAM))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        check(lib().qd_mlp_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), NPARAM))

    def forward(self, X, y, stream=None) -> None:
        check(lib().qd_mlp_forward(self.h, _ptr(X), _ptr(y), X.shape[0], C.c_void_p(stream)))

    def grad(self, X, T, g, stream=None) -> float:
        loss = C.c_float()
        check(lib().qd_mlp_grad(self.h, _ptr(X), _ptr(T), X.shape[0], _ptr(g), C.byref(loss), C.c_void_p(stream)))
        return loss.value

    def train_step(self, X, T, lr: float, stream=None, want_loss: bool = False):
        loss = C.c_float()
        check(lib().qd_mlp_train_step(self.h, _ptr(X), _ptr(T), X.shape[0], float(lr),
                                      C.byref(loss) if want_loss else None, C.c_void_p(stream)))
        return loss.value if want_loss else None

    def close(self) -> None:
        if getattr(self, "h", None) and self.h.value:
            lib().qd_mlp_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
class Instance:
    """One (N, R, hbar-omega) problem: HF Hamiltonian on the device."""

    def __init__(self, nbody: int, emax: int, hw: float, device: int = 0, mix: float = 0.5, quad: bool = True):
        vec, eig, _ = hf_hamiltonian(nbody, emax, hw, mix=mix, quad=quad)
        self.nbody, self.emax, self.hw = nbody, emax, hw
        self.P = Layout(nbody, emax, eig=eig, device=device)
        # the library's kernels and the torch buffers share torch's stream
        self.P.set_stream(_torch().cuda.current_stream().cuda_stream)
        self.H = FullHam(self.P, 1, vec)
        self.E_HF = float(vec[0])
        self.n = omega_count(self.P)
        self.crit0 = abs(mbpt2(self.H))
        torch = _torch()
        eta = FullHam(self.P, -1)
        build_white(eta, self.H)
        self.eta0 = torch.empty(self.n, dtype=torch.float64, device="cuda")
        omega_gather(eta, self.eta0)
        eta.close()

    def close(self):
        self.H.close()
        self.P.close()


def trajectory(inst: Instance, nsample: int, rng, max_iter: int = 300):
    """Run the plain flow, recording Omega on a fixed subset of
    entries after every accepted step.  Returns (idx [k], s [steps],
    omega [steps, k], result).  The subset is half uniform, half the entries
    of largest |Omega| at the first step (where the flow does most work)."""
    torch = _torch()
    HS = FullHam(inst.P, 1)
    f = Flow(inst.H, HS)
    buf = torch.empty(inst.n, dtype=torch.float64, device="cuda")
    snaps, svals, idx = [], [], None
    for _ in range(max_iter + 1):
        info = f.step()
        if info.accepted:
            omega_gather(f.omega(), buf)
            if idx is None:
                k = min(nsample, inst.n)
                top = torch.topk(buf.abs(), k // 2).indices
                uni = torch.from_numpy(rng.choice(inst.n, k - k // 2, replace=False)).to(buf.device)
                idx = torch.unique(torch.cat([top, uni]))
            snaps.append(buf[idx].float().clone())
            svals.append(info.s)
        if info.converged:
            break
    res = f.state()
    f.close()
    HS.close()
    return idx, np.array(svals), torch.stack(snaps), res


def samples(inst: Instance, idx, svals, omegas):
    """Training rows: features of the recorded entries at each recorded s,
    target r = Omega / eta0 (entries with |eta0| >= ETA_FLOOR, clipped)."""
    torch = _torch()
    X0 = torch.empty((inst.n, NFEAT), dtype=torch.float32, device="cuda")
    omega_features(inst.H, inst.hw, 0.0, X0)
    eta = inst.eta0[idx]
    keep = eta.abs() >= ETA_FLOOR
    base, eta = X0[idx][keep], eta[keep]
    xs, ts = [], []
    for s, om in zip(svals, omegas):
        x = base.clone()
        x[:, 13] = float(s) / 10.0
        xs.append(x)
        ts.append((om[keep].double() / eta).clamp(-RATIO_CLAMP, RATIO_CLAMP).float())
    return torch.cat(xs), torch.cat(ts)


def train(mlp: MLP, X, T, steps: int, batch: int = 8192, lr: float = 1e-3, seed: int = 0, log_every: int = 0):
    """Adam on random minibatches (rows drawn with a seeded generator); the
    learning rate decays by 10x over the run.  Returns the loss history."""
    torch = _torch()
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    batch = (batch // 32) * 32
    hist = []
    for k in range(steps):
        sel = torch.randint(0, X.shape[0], (batch,), device="cuda", generator=g)
        xb, tb = X[sel].contiguous(), T[sel].contiguous()
        want = log_every and (k % log_every == 0 or k == steps - 1)
        rate = lr * (0.1 ** (k / max(1, steps - 1)))
        loss = mlp.train_step(xb, tb, rate, want_loss=bool(want))
        if want:
            hist.append((k, loss))
    return hist


def predict_omega(mlp: MLP, inst: Instance, s: float) -> FullHam:
    """Omega predicted at flow parameter s, as a device operator."""
    torch = _torch()
    X = torch.empty((inst.n, NFEAT), dtype=torch.float32, device="cuda")
    omega_features(inst.H, inst.hw, s, X)
    y = torch.empty(inst.n, dtype=torch.float32, device="cuda")
    mlp.forward(X, y)
    G = FullHam(inst.P, -1)
    omega_scatter(G, y, 1.0, inst.eta0)
    torch.cuda.synchronize()
    return G


def cold_flow(inst: Instance, max_iter: int = 300):
    torch = _torch()
    HS = FullHam(inst.P, 1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f = Flow(inst.H, HS)
    r = f.run(max_iter)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    out = {"E": r.E0, "steps": r.iterations, "commutators": r.commutators, "seconds": dt, "s": r.s}
    f.close()
    HS.close()
    return out


def warm_flow(mlp: MLP, inst: Instance, s_target: float, max_iter: int = 300, window: int = 4,
              drop: float = 0.5):
    """The plain flow from the predicted Omega(s_target).  The prediction is
    judged by the flow itself and abandoned (the flow restarts from
    Omega = 0, its work counted) if the predicted state is not better than
    the HF start (|MBPT2| not below its s = 0 value), if the continued flow
    rejects a step (a rejection shrinks the Euler step for the rest of the
    flow, stp -> stp/2 + 1e-3, as s_evolve does) or if |MBPT2| falls by less
    than `drop` over `window` accepted steps.  The last two mean that the
    prediction seeded a slow mode: such flows can take several times the
    steps of the plain one (whose |MBPT2| falls about 10x over four steps)."""
    torch = _torch()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    G = predict_omega(mlp, inst, s_target)
    HS = FullHam(inst.P, 1)
    f = Flow(inst.H, HS)
    f.warm_start(G, s_target)
    info = f.step()
    crit_warm = float(info.crit)
    accepted = crit_warm < inst.crit0 and bool(info.accepted or info.converged)
    hist = [crit_warm]
    while accepted and not info.converged:
        info = f.step()
        if not info.accepted and not info.converged:
            accepted = False
        elif info.accepted:
            hist.append(float(info.crit))
            if len(hist) > window and hist[-1] > drop * hist[-1 - window]:
                accepted = False
    wasted = 0
    if accepted:
        r = f.state()
    else:
        wasted = f.state().commutators
        f.close()
        f = Flow(inst.H, HS)
        r = f.run(max_iter)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    out = {"E": r.E0, "steps": r.iterations, "commutators": r.commutators + wasted, "seconds": dt,
           "accepted": bool(accepted), "crit_warm": crit_warm, "crit0": inst.crit0, "wasted_commutators": wasted}
    f.close()
    HS.close()
    G.close()
    return out
