"""Interface calibration with a learned surrogate pre-screen (the reference's CMA-ES search,
flyzero/tune.py:26-166, scaled to 12 parameters and 1,024 candidates per generation).

The reference evaluates every candidate interface with a full race (emulator + brain). No
emulator exists here, so a candidate is judged on what the brain itself does: the interface maps
12 unit-box parameters to the Poisson drive of the T4/T5 stand-ins (a drifting grating seen
through a gain, a visible window, spatial and temporal frequency, direction, contrast, a rate cap,
a left/right balance) plus the tonic DNp09 drive, and the fitness of an episode of frames rewards
forward drive and balanced steering in the 10 readout descending neurons (DNs):

    fitness = mean over frames of [ c_fwd + 0.25 * sum(c_steer) - 0.5 * |c_left - c_right| ]

with c_fwd the DNp09 stand-in's count, c_left / c_right the first / last four motor DNs.

Per generation: the surrogate (flyzero_b200.surrogate.MLP) predicts the DN counts of all 1,024
candidates' episodes (autoregressively: each frame's features include the previous frame's
predicted counts); the best 64 are re-run on the full LIF engine at B=64, which judges the
surrogate (relative error of the episodes' DN counts, after a per-DN calibration learnt from the
previous survivors). CMA-ES is told the exact fitness of the 64
and the predicted fitness of the rest while that error is within tolerance, and only the 64 exact
values otherwise (the simulation is the fallback).

    python -m flyzero_b200.tuning --frames 200000 --generations 8
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import workloads as wl

SPACE12 = [
    ("log_gain", 1.3, 2.6),       # log10 of the grating's mean rate (Hz)
    ("y_min", 0.0, 0.7),          # fraction of the field (from the top) the fly ignores
    ("x_min", 0.0, 0.5),          # left edge of the visible window
    ("x_span", 0.3, 1.0),         # width of the visible window
    ("spatial_freq", 1.0, 8.0),   # cycles per field
    ("temporal_hz", 0.5, 6.0),
    ("direction", 0.0, 2 * np.pi),
    ("contrast", 0.2, 1.0),
    ("rate_cap", 50.0, 300.0),    # Hz
    ("drive_hz", 30.0, 150.0),    # tonic DNp09 drive
    ("balance", -0.5, 0.5),       # right-half gain minus left-half gain
    ("tonic_frac", 0.0, 1.0),     # share of the drive that is tonic (flat) rather than modulated
]
N_PARAMS = len(SPACE12)
PATCH_GRID = 32                   # 32 x 32 = 1,024 retinotopic patches
PROJ = 256


def unit_to_params(x):
    """(N, 12) unit-box rows -> (N, 12) parameter values (torch or numpy)."""
    lo = np.array([s[1] for s in SPACE12], np.float32)
    hi = np.array([s[2] for s in SPACE12], np.float32)
    try:
        import torch

        if isinstance(x, torch.Tensor):
            return torch.as_tensor(lo, device=x.device) + x * torch.as_tensor(hi - lo, device=x.device)
    except ImportError:
        pass
    return lo + np.asarray(x, np.float32) * (hi - lo)


def interface_rates(x, xy, t_ms: float):
    """Poisson rates (N, n_inputs + 1) of candidates x (N, 12) (torch, any device): the T4/T5
    stand-ins at positions xy (n_inputs, 2), then the tonic DNp09 drive."""
    import torch

    p = unit_to_params(x)
    gain = 10.0 ** p[:, 0:1]
    y_min, x_min, x_span = p[:, 1:2], p[:, 2:3], p[:, 3:4]
    sf, tf, th, con = p[:, 4:5], p[:, 5:6], p[:, 6:7], p[:, 7:8]
    cap, drive, bal, tonic = p[:, 8:9], p[:, 9:10], p[:, 10:11], p[:, 11:12]
    px, py = xy[:, 0][None, :], xy[:, 1][None, :]
    proj = px * torch.cos(th) + py * torch.sin(th)
    wave = torch.sin(2 * np.pi * (sf * proj - tf * (t_ms / 1000.0)))
    r = gain * (tonic + (1 - tonic) * (1 + con * wave))
    r = r * (1 + bal * torch.sign(px - 0.5))
    visible = (py >= y_min) & (px >= x_min) & (px <= x_min + x_span)
    r = torch.where(visible, torch.clamp(r, min=0.0), torch.zeros_like(r))
    r = torch.minimum(r, cap)
    return torch.cat([r, drive], dim=1).float()


def fitness(counts):
    """Episode fitness of DN counts (N, frames, 10) (numpy)."""
    c = np.asarray(counts, np.float64)
    fwd = c[:, :, 8]
    left, right = c[:, :, 0:4].sum(2), c[:, :, 4:8].sum(2)
    return (fwd + 0.25 * (left + right) - 0.5 * np.abs(left - right)).mean(1)


class Featurizer:
    """Frame inputs of the surrogate: log1p of the expected T4/T5 input spike counts binned to
    32 x 32 retinotopic patches, and a fixed 256-d projection of log1p(previous DN counts)."""

    def __init__(self, xy, device, seed: int = 0):
        import torch

        xy = np.asarray(xy)
        cell = np.minimum((xy * PATCH_GRID).astype(np.int64), PATCH_GRID - 1)
        patch = cell[:, 1] * PATCH_GRID + cell[:, 0]
        # deterministic binning: inputs sorted by patch, prefix sums read at the patch boundaries
        order = np.argsort(patch, kind="stable")
        ends = np.searchsorted(patch[order], np.arange(PATCH_GRID * PATCH_GRID), side="right")
        self.order = torch.as_tensor(order, device=device)
        self.ends = torch.as_tensor(ends, device=device)
        g = np.random.default_rng(seed + 99991)
        self.P = torch.as_tensor((g.standard_normal((PROJ, 10)) / np.sqrt(10)).astype(np.float32), device=device)
        self.n_in = len(xy)
        self.device = device

    def __call__(self, rates, prev_counts, window_ms: float = wl.FRAME_MS):
        import torch

        exp_in = rates[:, :self.n_in] * (window_ms / 1000.0)
        cum = torch.nn.functional.pad(exp_in.index_select(1, self.order).double().cumsum(1), (1, 0))
        sums = cum.index_select(1, self.ends)
        patches = torch.diff(sums, dim=1, prepend=cum[:, :1]).float().clamp(min=0.0)
        return torch.cat([torch.log1p(patches), torch.log1p(prev_counts) @ self.P.T], dim=1).contiguous()


class Simulator:
    """The full LIF engine running up to `batch` candidate interfaces side by side (B=64)."""

    def __init__(self, conn, drive, batch: int = 64, seed: int = 0):
        import torch

        from .brain import LIFParams
        from .gpu import BatchBrain

        self.gb = BatchBrain(conn.weights, LIFParams(dt=0.1), batch=batch, seed=seed)
        self.drive = drive
        self.B = batch
        idx_in = np.r_[drive.inputs, drive.tonic]
        self.cols = self.gb.slots(idx_in)
        self.readout = torch.as_tensor(drive.readout, device=self.gb.device)
        self.xy = torch.as_tensor(drive.xy.astype(np.float32), device=self.gb.device)
        self.scale = np.float32(0.1 / 1000.0)
        self.sims = 0

    def episode(self, x, frames: int, featurizer=None):
        """DN counts (N, frames, 10) of candidates x (N <= B, 12) from rest; with a featurizer also
        the surrogate's inputs (N, frames, 1280) and targets of every frame (teacher forcing)."""
        import torch

        gb = self.gb
        N = x.shape[0]
        xs = torch.zeros((self.B, N_PARAMS), device=gb.device)
        xs[:N] = torch.as_tensor(np.asarray(x, np.float32), device=gb.device)
        gb.reset()
        prev = torch.zeros((self.B, 10), device=gb.device)
        out = torch.empty((self.B, frames, 10), device=gb.device)
        feats = torch.empty((self.B, frames, 1280), device=gb.device) if featurizer else None
        counts = torch.empty((self.B, gb.n), dtype=torch.int32, device=gb.device)
        for f in range(frames):
            rates = interface_rates(xs, self.xy, f * wl.FRAME_MS)
            gb.p_ext[:, self.cols] = rates * torch.tensor(self.scale, device=gb.device)
            if featurizer is not None:
                feats[:, f] = featurizer(rates, prev)
            gb.run_steps(wl.frame_steps(0.1), counts=counts)
            dn = counts.index_select(1, self.readout).float()
            out[:, f] = dn
            prev = dn
        self.sims += N
        return (out[:N], feats[:N] if featurizer else None)


def generate_frames(sim: Simulator, feat: Featurizer, n_frames: int, episode: int = 30, seed: int = 0):
    """Training frames from the simulator: random interfaces, `episode` frames each from rest."""
    import torch

    rng = np.random.default_rng(seed)
    Xs, Ys = [], []
    have = 0
    while have < n_frames:
        x = rng.random((sim.B, N_PARAMS)).astype(np.float32)
        dn, feats = sim.episode(x, episode, featurizer=feat)
        Xs.append(feats.reshape(-1, 1280))
        Ys.append(dn.reshape(-1, 10))
        have += sim.B * episode
    X = torch.cat(Xs)[:n_frames].contiguous()
    Y = torch.cat(Ys)[:n_frames].contiguous()
    return X, Y


def train(net, X, Y, epochs: int, batch: int = 4096, seed: int = 0):
    """Mini-batch training; returns per-epoch mean losses."""
    import torch

    g = torch.Generator(device=X.device).manual_seed(seed)
    losses = []
    for _ in range(epochs):
        perm = torch.randperm(X.shape[0], device=X.device, generator=g)
        tot, nb = 0.0, 0
        for k in range(0, X.shape[0] - batch + 1, batch):
            sel = perm[k:k + batch]
            tot += net.train_step(X[sel].contiguous(), Y[sel].contiguous())
            nb += 1
        losses.append(float(tot / max(nb, 1)))
    return losses


def surrogate_episode(net, feat, xy, x, frames: int, cap=None):
    """Predicted expected DN counts (N, frames, 10) of candidates x (N, 12) (torch on the GPU). The
    rollout feeds each frame's prediction back as the next frame's previous counts; `cap` (10,),
    the largest count of each DN in the simulated frames, bounds what is fed back and predicted, so
    that an overrated frame cannot run away outside the range the network was trained on."""
    import torch

    xs = torch.as_tensor(np.asarray(x, np.float32), device=feat.device)
    prev = torch.zeros((xs.shape[0], 10), device=feat.device)
    out = torch.empty((xs.shape[0], frames, 10), device=feat.device)
    for f in range(frames):
        X = feat(interface_rates(xs, xy, f * wl.FRAME_MS), prev)
        mu = torch.exp(net.forward(X).clamp(-20.0, 8.0))      # bounded: predictions feed back
        if cap is not None:
            mu = torch.minimum(mu, cap)
        out[:, f] = mu
        prev = mu
    return out


def count_error(pred, true):
    """Relative error of each episode's total DN count, (N,) numpy (includes the Poisson noise of
    the single simulated episode)."""
    p = np.asarray(pred, np.float64).sum((1, 2))
    t = np.asarray(true, np.float64).sum((1, 2))
    return np.abs(p - t) / np.maximum(t, 1.0)


def aggregate_count_error(pred, true):
    """Relative error of the DN counts summed over a set of episodes, averaged over the DNs
    (weighted by their counts): the surrogate's bias on the simulated set."""
    p = np.asarray(pred, np.float64).sum((0, 1))
    t = np.asarray(true, np.float64).sum((0, 1))
    return float(np.abs(p - t).sum() / max(t.sum(), 1.0))


def search_with_surrogate(net, feat, sim, generations: int, popsize: int = 1024, survivors: int = 64,
                          frames: int = 30, tol: float = 0.05, seed: int = 0, data=None, refine_steps: int = 20):
    """Surrogate-screened CMA-ES. The survivors' simulated frames also refine the surrogate
    (`refine_steps` Adam steps on them mixed with the original training frames `data`), and a
    per-DN calibration factor (simulated counts over the refined network's predicted counts on the
    same survivors) corrects what bias the network keeps: picking the best of 1,024 predictions
    picks the ones the network overrates, so its raw error on the survivors exceeds its error on
    the training distribution."""
    import torch

    from .cmaes import CMAES

    es = CMAES(np.full(N_PARAMS, 0.5), 0.3, popsize, seed=seed)
    best, log = -np.inf, []
    g_rng = torch.Generator(device=feat.device).manual_seed(seed)
    newX, newY = [], []
    scale = np.ones(10)                          # per-DN calibration of the predicted counts
    cap = data[1].amax(0).float() if data is not None else None
    for g in range(generations):
        X = es.ask()
        raw = surrogate_episode(net, feat, sim.xy, X, frames, cap).cpu().numpy()
        pc = raw * scale
        pf = fitness(pc)
        top = np.argsort(-pf, kind="stable")[:survivors]
        tc_d, tfeat = sim.episode(X[top], frames, featurizer=feat)
        tc = tc_d.cpu().numpy()
        tf = fitness(tc)
        err = aggregate_count_error(pc[top], tc)
        err_raw = aggregate_count_error(raw[top], tc)
        per = float(np.mean(count_error(pc[top], tc)))
        newX.append(tfeat.reshape(-1, 1280))
        newY.append(tc_d.reshape(-1, 10))
        cap = newY[-1].amax(0).float() if cap is None else torch.maximum(cap, newY[-1].amax(0).float())
        if refine_steps and data is not None:
            NX, NY = torch.cat(newX), torch.cat(newY)
            for _ in range(refine_steps):
                i_new = torch.randint(0, NX.shape[0], (2048,), device=feat.device, generator=g_rng)
                i_old = torch.randint(0, data[0].shape[0], (2048,), device=feat.device, generator=g_rng)
                net.train_step(torch.cat([NX[i_new], data[0][i_old]]).contiguous(),
                               torch.cat([NY[i_new], data[1][i_old]]).contiguous())
        # calibration for the next generation: the refined network on these survivors
        again = surrogate_episode(net, feat, sim.xy, X[top], frames, cap).cpu().numpy()
        scale = tc.sum((0, 1)) / np.maximum(again.sum((0, 1)), 1e-6)
        scale = np.clip(np.where(tc.sum((0, 1)) > 0, scale, 1.0), 0.25, 4.0)   # a DN predicted silent: bounded
        if err <= tol:
            f_all = pf.copy()
            f_all[top] = tf
            es.tell(X, -f_all)
        else:
            es.tell(X[top], -tf)
        best = max(best, float(tf.max()))
        log.append({"gen": g, "screened": popsize, "simulated": survivors, "count_error": err,
                    "count_error_uncalibrated": err_raw, "count_error_per_episode": per, "within_tol": err <= tol,
                    "best_true": float(tf.max()), "best_so_far": best,
                    "fitness_error": float(np.mean(np.abs(pf[top] - tf)) / max(np.mean(np.abs(tf)), 1e-9))})
    return best, log


def search_plain(sim, generations: int, popsize: int = 64, frames: int = 30, seed: int = 0):
    """CMA-ES without the surrogate: every candidate of every generation is simulated."""
    from .cmaes import CMAES

    es = CMAES(np.full(N_PARAMS, 0.5), 0.3, popsize, seed=seed)
    best, log = -np.inf, []
    for g in range(generations):
        X = es.ask()
        tc, _ = sim.episode(X, frames)
        tf = fitness(tc.cpu().numpy())
        es.tell(X, -tf)
        best = max(best, float(tf.max()))
        log.append({"gen": g, "simulated": popsize, "best_true": float(tf.max()), "best_so_far": best})
    return best, log


def run(n: int = 138_639, frames: int = 200_000, epochs: int = 12, generations: int = 8, episode: int = 30,
        seed: int = 0) -> dict:
    import torch

    from . import connectome as cx
    from .surrogate import MLP

    conn = cx.flywire_scale() if n == 138_639 else cx.synthetic(n, seed=seed, motor=8, motor_in=min(7300, n))
    n_in = 12_246 if n == 138_639 else max(256, n // 12)
    drive = wl.grating_drive(conn.n, seed=seed, n_inputs=n_in, exclude=conn.motor)
    sim = Simulator(conn, drive, batch=64, seed=seed)
    feat = Featurizer(drive.xy, sim.gb.device, seed=seed)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    X, Y = generate_frames(sim, feat, frames, episode=episode, seed=seed)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t0
    n_val = max(4096, frames // 10)
    Xv, Yv, Xt, Yt = X[:n_val], Y[:n_val], X[n_val:], Y[n_val:]
    net = MLP(seed=seed)
    t0 = time.perf_counter()
    losses = train(net, Xt, Yt, epochs)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    steps = epochs * (Xt.shape[0] // 4096)
    flops = steps * 4096 * 3 * 2 * (1280 * 512 + 512 * 512 + 512 * 10)
    net.forward(Xv, training=True)
    val = float(net.backward(Yv))
    mu = torch.exp(net.forward(Xv))
    val_err = float((mu.sum() - Yv.sum()).abs() / Yv.sum())
    mean_counts = Yv.mean(0).cpu().numpy().tolist()
    sims0 = sim.sims
    t0 = time.perf_counter()
    best_s, log_s = search_with_surrogate(net, feat, sim, generations, frames=episode, seed=seed + 1, data=(Xt, Yt))
    t_s = time.perf_counter() - t0
    sims_s = sim.sims - sims0
    sims0 = sim.sims
    best_p, log_p = search_plain(sim, generations, frames=episode, seed=seed + 1)
    sims_p = sim.sims - sims0
    return {"n": conn.n, "frames": frames, "gen_seconds": t_gen, "frames_per_s": frames / t_gen,
            "train": {"epochs": epochs, "steps": steps, "seconds": t_train, "tflops": flops / t_train / 1e12,
                      "loss_per_epoch": losses, "val_nll": val, "val_total_count_error": val_err,
                      "mean_dn_counts": mean_counts},
            "surrogate_search": {"best": best_s, "sims": sims_s, "seconds": t_s, "log": log_s},
            "plain_search": {"best": best_p, "sims": sims_p, "log": log_p}}


def main(argv=None):
    ap = argparse.ArgumentParser(description="surrogate-screened interface calibration")
    ap.add_argument("--n", type=int, default=138_639)
    ap.add_argument("--frames", type=int, default=200_000)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--generations", type=int, default=8)
    ap.add_argument("--episode", type=int, default=30)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    print(json.dumps(run(a.n, a.frames, a.epochs, a.generations, a.episode, a.seed)))


if __name__ == "__main__":
    main()
