"""The learned-closure workload: data from a fine DNS, training, and the
coarse closed run compared with a held-out DNS.

    python -m tara2d_b200.closure_run train    --out DIR [options]
    python -m tara2d_b200.closure_run evaluate --out DIR [options]

train: for each training seed, an FP64 MHD DNS on N x N (nu = eta = 1e-4,
CS = 100, random-phase u and B with E(k) ~ k^4 exp(-(k/k0)^2)) is spun up and
then sampled every `--pair-every` steps; each sample is sharp-filtered to
Nc x Nc and turned into an (input, subgrid stress/EMF) pair on the device.
With `--ensemble M` the pairs come instead from M fine runs (N <= 512)
stepped together as one batched ensemble (AB2 at `--ensemble-dt`, sampled at
the same model times), one pair per member per sample, until `--capacity`.
The CNN is trained on the pairs and saved with its normalisation to
DIR/closure_model.npz.

evaluate: a held-out seed is run as a DNS to time T (its E(k) and device time
recorded), and its filtered initial state is run on Nc x Nc without the
closure, with it at every RK4 stage, and with it once per step (dt scaled by
N/Nc).  Writes DIR/closure_eval.json: E(k) of the runs for k <= kmax, the
worst relative E(k) error of each coarse run, and the device-time ratios
DNS / closed run.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import (CLOSURE_EVERY_RHS, CLOSURE_ONCE_PER_STEP, FP64, MODEL_COM, STEP_RK4, Closure, Params, Session,
               attach_closure, filter_state, initial)

PI = 3.14159265358979323846


def params(nu, dt):
    return Params.make(Lx=2 * PI, Ly=2 * PI, pi=PI, dt=dt, mu=nu, eta=nu, CS=100.0, spheat=5.0 / 3.0, ms=1.0,
                       mu_0=1.0, kf=1.0, A=0.0, fix_curlB=0)


def dns_session(N, seed, k0, nu, dt):
    s = Session(MODEL_COM, N, N, params(nu, dt), precision=FP64)
    s.set_state(initial.com_random_phase(N, N, seed=seed, k0=k0))
    return s


def ensemble_pairs(a, c):
    """Training pairs from an FP64 MHD ensemble of `a.ensemble` fine runs
    (seeds train_seeds[0], train_seeds[0] + 1, ...) stepped together by AB2
    at dt = `a.ensemble_dt` (ensembles step with AB2; at CS = 100 AB2 needs a
    smaller dt than RK4), spun up and sampled at the model times of the
    RK4 schedule; each sample gives one pair per member.  Returns the
    ensemble's AB2 steps."""
    from . import STEP_AB2, Ensemble
    M = a.ensemble
    spin = max(1, round(a.spin_steps * a.dt / a.ensemble_dt))
    every = max(1, round(a.pair_every * a.dt / a.ensemble_dt))
    steps = 0
    with Ensemble([a.n] * M, params(a.nu, a.ensemble_dt), precision=FP64, model=MODEL_COM) as e:
        for m in range(M):
            e.set_state(m, initial.com_random_phase(a.n, a.n, seed=a.train_seeds[0] + m, k0=a.k0))
        e.step(STEP_AB2, spin)
        steps += spin
        while c.count + M <= a.capacity:
            e.step(STEP_AB2, every)
            steps += every
            for m in range(M):
                c.add_pair_member(e, m)
    return steps


def train(a):
    c = Closure(a.nc, a.capacity, batch_max=a.batch, seed=a.seed)
    t0 = time.time()
    dns_ms = 0.0
    ens_steps = 0
    if a.ensemble:
        ens_steps = ensemble_pairs(a, c)
    else:
        for seed in a.train_seeds:
            with dns_session(a.n, seed, a.k0, a.nu, a.dt) as s:
                dns_ms += s.time_steps(STEP_RK4, a.spin_steps)
                for _ in range(a.pairs_per_seed):
                    if c.count >= a.capacity:
                        break
                    dns_ms += s.time_steps(STEP_RK4, a.pair_every)
                    c.add_pair(s)
    npairs = c.count
    nval = max(1, npairs // 10)
    ntrain = npairs - nval
    c.fit_norm(0, ntrain)
    loss0 = c.eval_loss(0, ntrain)
    val0 = c.eval_loss(ntrain, nval)
    t1 = time.time()
    losses = []
    lr = a.lr
    for ep in range(a.epochs):
        if ep and ep % max(1, a.epochs // 3) == 0:
            lr *= 0.3
        losses += list(map(float, c.train(0, ntrain, 1, batch=a.batch, lr=lr)))
    t2 = time.time()
    val1 = c.eval_loss(ntrain, nval)
    np.savez(os.path.join(a.out, "closure_model.npz"), params=c.get_params(), norm=c.get_norm())
    rep = {"pairs": npairs, "train_pairs": ntrain, "validation_pairs": nval, "grid": [a.n, a.nc],
           "source": f"ensemble of {a.ensemble} members, AB2 dt {a.ensemble_dt}" if a.ensemble else "sessions",
           "ensemble_steps": ens_steps,
           "dns_device_s": dns_ms / 1e3, "data_wall_s": t1 - t0, "train_wall_s": t2 - t1, "epochs": a.epochs,
           "loss_before": loss0, "validation_before": val0, "epoch_loss": losses, "validation_after": val1}
    with open(os.path.join(a.out, "closure_train.json"), "w") as f:
        json.dump(rep, f, indent=1)
    c.close()
    return rep


def _errors(res, name, ek_final, ek_avg, dns_final, dns_avg, kmax):
    ks = np.arange(1, kmax + 1)
    for tag, ek, ref in (("final", ek_final, dns_final), ("window", ek_avg, dns_avg)):
        rel = np.abs(np.asarray(ek[1:kmax + 1]) - ref[1:kmax + 1]) / ref[1:kmax + 1]
        ok = bool(np.all(np.isfinite(rel)))
        res[f"{name}_{tag}_max_rel_err"] = float(np.max(rel)) if ok else None
        res[f"{name}_{tag}_worst_k"] = int(ks[np.argmax(rel)]) if ok else None
        res[f"{name}_{tag}_within_5pct_up_to_k"] = int(np.argmax(np.append(rel, 1.0) > 0.05)) if ok else 0
        res[f"{name}_{tag}_rel_err"] = rel.tolist()


def evaluate(a):
    """E(k) at the final time and averaged over the records of the second half
    of the run (every `rec_every` fine steps), for the DNS, the unclosed and
    the closed coarse runs (the closure at every RK4 stage, and once per
    step: "closed_once"); device times of the runs."""
    m = np.load(a.model or os.path.join(a.out, "closure_model.npz"))
    c = Closure(a.nc, 1, batch_max=1)
    c.set_params(m["params"])
    c.set_norm(m["norm"])
    ratio = a.n // a.nc
    fine_steps = a.eval_steps - a.eval_steps % a.rec_every
    nrec = fine_steps // a.rec_every + 1
    half = nrec // 2
    res, spectra = {}, {}
    kmax = a.kmax
    with dns_session(a.n, a.eval_seed, a.k0, a.nu, a.dt) as fine:
        with Session(MODEL_COM, a.nc, a.nc, params(a.nu, a.dt * ratio)) as co:
            filter_state(fine, co)
            coarse_ic = co.get_state()
        _, ek = fine.run_recorded(STEP_RK4, a.rec_every, nrec)
        dns_final, dns_avg = ek[-1], ek[half:].mean(axis=0)
        res["dns_ms"] = fine.time_steps(STEP_RK4, 2000) / 2000 * fine_steps  # pure stepping, scaled
    spectra["dns_final"], spectra["dns_window"] = dns_final[:kmax + 1].tolist(), dns_avg[:kmax + 1].tolist()
    for name, closed, mode in (("coarse", False, CLOSURE_EVERY_RHS), ("closed", True, CLOSURE_EVERY_RHS),
                               ("closed_once", True, CLOSURE_ONCE_PER_STEP)):
        with Session(MODEL_COM, a.nc, a.nc, params(a.nu, a.dt * ratio)) as co:
            co.set_state(coarse_ic)
            if closed:
                co.set_closure_mode(mode)
                attach_closure(co, c)
            try:
                _, ek = co.run_recorded(STEP_RK4, a.rec_every // ratio, nrec)
                co.set_state(coarse_ic)
                res[name + "_ms"] = co.time_steps(STEP_RK4, fine_steps // ratio)
            except Exception as e:  # a run that blows up is a result, not a crash of the workload
                ek = np.full((nrec, kmax + 1), np.nan)
                res[name + "_ms"] = None
                res[name + "_error"] = str(e)
            if closed:
                attach_closure(co, None)
        fin, avg = ek[-1], ek[half:].mean(axis=0)
        spectra[name + "_final"], spectra[name + "_window"] = fin[:kmax + 1].tolist(), avg[:kmax + 1].tolist()
        _errors(res, name, fin, avg, dns_final, dns_avg, kmax)
    res["time"] = fine_steps * a.dt
    res["window"] = [half * a.rec_every * a.dt, fine_steps * a.dt]
    res["speedup_dns_over_closed"] = res["dns_ms"] / res["closed_ms"] if res.get("closed_ms") else None
    res["speedup_dns_over_closed_once"] = (res["dns_ms"] / res["closed_once_ms"]
                                           if res.get("closed_once_ms") else None)
    res["spectra"] = spectra
    with open(os.path.join(a.out, "closure_eval.json"), "w") as f:
        json.dump(res, f, indent=1)
    c.close()
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("stage", choices=["train", "evaluate"])
    ap.add_argument("--out", required=True)
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--nc", type=int, default=256)
    ap.add_argument("--nu", type=float, default=1e-4)
    ap.add_argument("--k0", type=float, default=4.0)
    ap.add_argument("--dt", type=float, default=3.8e-5)  # CS kmax dt = 100 * 683 * 3.8e-5 = 2.6 < 2.83
    ap.add_argument("--train-seeds", type=int, nargs="+", default=[101, 102])
    ap.add_argument("--eval-seed", type=int, default=201)
    ap.add_argument("--spin-steps", type=int, default=20000)
    ap.add_argument("--pair-every", type=int, default=25)
    ap.add_argument("--pairs-per-seed", type=int, default=400)
    ap.add_argument("--capacity", type=int, default=800)
    ap.add_argument("--ensemble", type=int, default=0,
                    help="train: take the pairs from an ensemble of this many fine runs (N <= 512)")
    ap.add_argument("--ensemble-dt", type=float, default=1e-5, help="AB2 time step of the ensemble runs")
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--eval-steps", type=int, default=24000)
    ap.add_argument("--kmax", type=int, default=80)
    ap.add_argument("--rec-every", type=int, default=800)
    ap.add_argument("--model", default=None, help="closure_model.npz to evaluate (default: OUT/closure_model.npz)")
    a = ap.parse_args(argv)
    os.makedirs(a.out, exist_ok=True)
    rep = train(a) if a.stage == "train" else evaluate(a)
    print(json.dumps({k: v for k, v in rep.items() if not isinstance(v, (list, dict))}), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
