"""Learned warm start: training data from the plain solver, training on the
GPU with the library's own kernels, evaluation, and the weights file.

    python -m chysx.learned train --out chysx/data/warmstart.npz
    python -m chysx.learned eval  --net chysx/data/warmstart.npz

Training distribution (seed 2): square grids with side U{64..128}, +-1%
jitter, per-edge spring k log-U[1e2,1e4], Baraff-Witkin k 1e4, 1-4 random
corner pins and a random constant wind force |f| ~ U[0, 2] N/m^2 (applied as
f_i = w * A_i with A_i the lumped area of vertex i).  Every solve runs the
plain zero-guess PCG to rel-res 1e-6; a sample is one vertex of one step:
the step's 20 features (exported by the simulator's feature tap) and the
target dv = v_{n+1} - v_n.  The network trained on it is evaluated on
held-out seeds of the 256x256 plain-method distribution, where the PCG still
runs to rel-res 1e-6 (zero guess as fallback), so only the iteration count
can change.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import capi, scenes

N_FEATURES = 20
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_NET = os.path.join(HERE, "data", "warmstart.npz")
FORMAT_VERSION = 1


def n_params() -> int:
    return int(capi.lib().chysx_mlp_num_params())


# ---------------------------------------------------------------------------
# weights file
# ---------------------------------------------------------------------------
def save(path, params, meta):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez_compressed(path, params=np.asarray(params, np.float32), version=np.int32(FORMAT_VERSION),
                        meta=json.dumps(meta))


def load(path=DEFAULT_NET):
    d = np.load(path)
    if int(d["version"]) != FORMAT_VERSION:
        raise ValueError(f"{path}: weights format {int(d['version'])}, expected {FORMAT_VERSION}")
    p = d["params"].astype(np.float32)
    if p.shape[0] != n_params():
        raise ValueError(f"{path}: {p.shape[0]} parameters, the library expects {n_params()}")
    return p, json.loads(str(d["meta"]))


# ---------------------------------------------------------------------------
# training scenes and data collection
# ---------------------------------------------------------------------------
def training_instances(rng, count, lo=64, hi=128):
    out = []
    for b in range(count):
        side = int(rng.integers(lo, hi + 1))
        pos, tris = scenes.grid_mesh(side)
        h = 1.0 / (side - 1)
        pos = pos + rng.uniform(-0.01 * h, 0.01 * h, pos.shape)
        E = scenes.unique_edges(tris).shape[0]
        k_spring = np.exp(rng.uniform(np.log(1e2), np.log(1e4), E)).astype(np.float32)
        corners = np.array([0, side - 1, (side - 1) * side, side * side - 1])
        pins = np.sort(rng.choice(corners, int(rng.integers(1, 5)), replace=False))
        sc = scenes._finish(f"train{b}_s{side}", pos, tris, k_spring, 1.0e4, pins, 0, 20000, 1e-6)
        d = rng.standard_normal(3)
        sc["wind"] = (d / np.linalg.norm(d) * rng.uniform(0.0, 2.0)).astype(np.float32)
        out.append(sc)
    return out


def collect(total_steps=20000, seed=2, batch=32, steps_per_scene=40, samples_per_step=256, log=print):
    """Runs plain-solver steps on packed batches of training scenes and
    returns (features, targets) as CUDA tensors."""
    import torch

    from .runner import GpuCloth

    rng = np.random.default_rng(seed)
    feats, targs = [], []
    done = 0
    t0 = time.time()
    while done < total_steps:
        insts = training_instances(rng, batch)
        sc, offs = scenes.concat(insts)
        n = sc["pos"].shape[0]
        sc["force"] = np.zeros((n, 3), np.float32)
        g = GpuCloth(sc, max_iter=20000, rel_tol=1e-6, warm_start="zero", apply_force=True, instances=offs)
        # wind force per vertex: w * lumped area (= mass / density)
        area = (1.0 / torch.clamp(g.inv_mass, min=1e-12)) / sc["density"]
        wind = torch.from_numpy(np.concatenate([np.repeat(s["wind"][None], s["pos"].shape[0], 0) for s in insts]))
        g.force.copy_(wind.cuda() * area[:, None])
        fbuf = torch.zeros((n, N_FEATURES), dtype=torch.float32, device="cuda")
        g.sim.set_feature_output(fbuf.data_ptr())
        inst_of = np.repeat(np.arange(len(insts)), np.diff(offs))
        for k in range(steps_per_scene):
            v_old = g.vel.clone()
            g.step()
            it, rr, st = g.sim.instance_stats()
            ok = np.flatnonzero((st == capi.SOLVE_CONVERGED) & (rr <= 1e-6))
            dv = g.vel - v_old
            for b in ok:
                lo, hi = int(offs[b]), int(offs[b + 1])
                idx = torch.from_numpy(rng.integers(lo, hi, samples_per_step)).cuda()
                feats.append(fbuf[idx].clone())
                targs.append(dv[idx].clone())
            done += len(ok)
            if done >= total_steps:
                break
        log(f"collect: {done}/{total_steps} instance-steps, {time.time() - t0:.1f}s")
        del g
    return torch.cat(feats), torch.cat(targs)


# ---------------------------------------------------------------------------
# training
# ---------------------------------------------------------------------------
def init_params(rng, mu_in, sd_in, mu_out, sd_out):
    """He initialisation with the standardisation statistics in front."""
    p = np.zeros(n_params(), np.float32)
    k = 0

    def put(v):
        nonlocal k
        v = np.asarray(v, np.float32).ravel()
        p[k:k + v.size] = v
        k += v.size

    put(mu_in)
    put(sd_in)
    put(mu_out)
    put(sd_out)
    for fan_in, fan_out in ((N_FEATURES, 64), (64, 64), (64, 64), (64, 3)):
        put(rng.standard_normal((fan_in, fan_out)) * np.sqrt(2.0 / fan_in))
        put(np.zeros(fan_out))
    assert k == p.size
    return p


class Trainer:
    """Adam on the FP32 master copy; forward/backward/weight-gradient kernels
    of the library (BF16 tensor cores, FP32 accumulation)."""

    def __init__(self, params, max_rows):
        import torch

        self.torch = torch
        self.p = torch.from_numpy(np.asarray(params, np.float32)).cuda()
        self.g = torch.zeros_like(self.p)
        self.m1 = torch.zeros_like(self.p)
        self.m2 = torch.zeros_like(self.p)
        self.max_rows = max_rows
        nbytes = int(capi.lib().chysx_mlp_workspace_bytes(max_rows))
        self.ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        self.t = 0

    def step(self, feats, targs, lr):
        import ctypes

        rows = feats.shape[0]
        assert rows <= self.max_rows
        self.t += 1
        loss = ctypes.c_double()
        capi.check(capi.lib().chysx_mlp_train_step(
            self.p.data_ptr(), self.g.data_ptr(), self.m1.data_ptr(), self.m2.data_ptr(), feats.data_ptr(),
            targs.data_ptr(), rows, lr, self.t, self.ws.data_ptr(), self.ws.numel(), ctypes.byref(loss), 0))
        return loss.value

    def loss(self, feats, targs):
        import ctypes

        loss = ctypes.c_double()
        capi.check(capi.lib().chysx_mlp_gradients(
            self.p.data_ptr(), feats.data_ptr(), targs.data_ptr(), feats.shape[0], self.g.data_ptr(),
            ctypes.byref(loss), self.ws.data_ptr(), self.ws.numel(), 0))
        return loss.value

    def params(self):
        return self.p.cpu().numpy()


def train(feats, targs, epochs=30, batch_rows=8192, lr=2e-3, seed=0, log=print):
    import torch

    rng = np.random.default_rng(seed)
    f64 = feats.double()
    t64 = targs.double()
    mu_in = f64.mean(0).cpu().numpy()
    sd_in = f64.std(0).clamp(min=1e-6).cpu().numpy()
    mu_out = t64.mean(0).cpu().numpy()
    sd_out = t64.std(0).clamp(min=1e-9).cpu().numpy()
    n = feats.shape[0]
    perm = torch.from_numpy(rng.permutation(n)).cuda()
    n_val = min(n // 10, 65536)
    val, tr = perm[:n_val], perm[n_val:]
    fv, tv = feats[val].contiguous(), targs[val].contiguous()
    trainer = Trainer(init_params(rng, mu_in, sd_in, mu_out, sd_out), max(batch_rows, n_val))
    history = []
    for ep in range(epochs):
        order = tr[torch.from_numpy(rng.permutation(tr.numel())).cuda()]
        lr_ep = lr * 0.5 * (1.0 + np.cos(np.pi * ep / epochs))
        tot, cnt = 0.0, 0
        for s in range(0, order.numel() - batch_rows + 1, batch_rows):
            idx = order[s:s + batch_rows]
            tot += trainer.step(feats[idx].contiguous(), targs[idx].contiguous(), lr_ep)
            cnt += 1
        vl = trainer.loss(fv, tv)
        history.append((ep, tot / max(cnt, 1), vl))
        log(f"epoch {ep}: train {tot / max(cnt, 1):.4f}  val {vl:.4f}")
    return trainer.params(), history


# ---------------------------------------------------------------------------
# evaluation: iterations to rel-res 1e-6, learned vs zero guess
# ---------------------------------------------------------------------------
def evaluate(params, seeds=(100, 101), steps=20, side=256,
             modes=("zero", "previous", "previous_scaled", "learned"), log=print):
    """PCG iterations per step to rel-res 1e-6 on held-out seeds of the
    256x256 configuration for each start mode (the zero guess is the
    reference point)."""
    from .runner import GpuCloth

    rows = []
    for seed in seeds:
        sc = scenes.config_large(side=side, seed=seed, max_iter=30000)
        res = {}
        for mode in modes:
            g = GpuCloth(sc, max_iter=30000, rel_tol=1e-6, warm_start="zero")
            if mode == "learned":
                g.sim.set_network(params)
            g.sim.set_solver(30000, 1e-6, mode)
            its, kept = [], 0
            for _ in range(steps):
                g.step()
                its.append(g.stats()[0])
                if mode != "zero":
                    kept += g.sim.guess_kept()
            res[mode] = (np.array(its), g.positions(), kept)
        z = res["zero"]
        row = dict(seed=seed, steps=steps, zero_iters=float(z[0].mean()))
        for mode in modes:
            if mode == "zero":
                continue
            m = res[mode]
            row[f"{mode}_iters"] = float(m[0].mean())
            row[f"{mode}_ratio"] = float(z[0].sum() / max(1, m[0].sum()))
            row[f"{mode}_guess_kept"] = int(m[2])
            row[f"{mode}_max_pos_diff"] = float(np.abs(z[1] - m[1]).max())
        log(json.dumps(row))
        rows.append(row)
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "eval"])
    ap.add_argument("--out", default=DEFAULT_NET)
    ap.add_argument("--net", default=DEFAULT_NET)
    ap.add_argument("--steps", type=int, default=20000, help="training instance-steps")
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--eval-steps", type=int, default=20)
    args = ap.parse_args()
    if args.cmd == "train":
        t0 = time.time()
        feats, targs = collect(total_steps=args.steps)
        t1 = time.time()
        params, hist = train(feats, targs, epochs=args.epochs)
        t2 = time.time()
        meta = dict(samples=int(feats.shape[0]), instance_steps=args.steps, seed=2, epochs=args.epochs,
                    collect_s=t1 - t0, train_s=t2 - t1, final_val_loss=hist[-1][2],
                    features="v, dt*g_ext, ring offset, ring dv, dt*a_el, dt*ring a_el, pinned, log10 k")
        save(args.out, params, meta)
        print(json.dumps(meta))
        print(json.dumps(evaluate(params, steps=args.eval_steps)))
    else:
        params, meta = load(args.net)
        print(json.dumps(evaluate(params, steps=args.eval_steps)))


if __name__ == "__main__":
    main()
