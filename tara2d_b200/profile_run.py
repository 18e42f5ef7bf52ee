"""Per-kernel timing of one session workload, for profiling runs.

    python -m tara2d_b200.profile_run --model com|coh|csh|css --grid N
        [--fp32] [--stepper rk4|ab2] [--steps K] [--warmup W]

Builds the seeded state of the model's benchmark configuration (hydro:
random phase + density noise, MHD: Orszag-Tang + 1e-3 perturbation on
8 <= |k| <= 16, both built on the device; vorticity: host random phase),
takes W warm-up steps, times K steps (CUDA events, graph replay), then
times every kernel of K more steps (an event before each launch, host
launches).  Prints one JSON line: steps/s and, per kernel, the mean launch
time, the algorithmic bytes of one launch (every field the kernel must read
or write, once; S = one spectral field in the session's precision) and their
ratio in GB/s.
"""
from __future__ import annotations

import argparse
import json
import sys

from . import (FP32, FP64, IC_ORSZAG_TANG, IC_RANDOM_PHASE, MODEL_COH, MODEL_COM, MODEL_CSH, MODEL_CSS, STEP_AB2,
               STEP_RK4, Params, Session, initial)

PI = 3.14159265358979323846
VPI = float(__import__("numpy").float32(3.1428))  # the vorticity units' default-real pi


def stepper_fields(stepper: int) -> float:
    """Stepper traffic per field per RHS, in S: AB2 reads u and the old
    derivative and writes the new state and derivative (4); RK4 averaged over
    its stages (3, 4, 4, 2)."""
    return 4.0 if stepper == STEP_AB2 else (3 + 4 + 4 + 2) / 4.0


def kernel_bytes(model: int, stepper: int, S: float) -> dict:
    st = stepper_fields(stepper)
    if model == MODEL_COM:
        return {"k_col_inv": 12 * S,          # 6 state fields in, 6 half-real out
                "k_row_com1": 14 * S,         # 6 in, 8 fluxes out
                "k_col_rt": 2 * S,            # X(uy) in, d(uy)/dy out
                "k_row_com2": 7 * S,          # 4 in, 3 energy-flux parts out
                # fluxes, stage input + stepper (RK4: 18/28/28/16 S over the stages,
                # as bench.py counts them; AB2: the stage input is the state), next y-inverse
                "k_col_fwd_com": (11 + ((18 + 28 + 28 + 16) / 4.0 if stepper == STEP_RK4 else 6 * st) + 6) * S}
    if model == MODEL_COH:
        return {"k_col_inv": 11 * S,          # 3 state fields in, 8 half-real out
                "k_row_coh": 11 * S,          # 8 in, 3 out
                "k_col_fwd_simple": (3 + 3 * st) * S}
    return {"k_col_inv": 5 * S,               # omega in, psi, i ky psi, W, i ky W out
            "k_row_vort": 5 * S,              # 4 in, 1 out
            "k_col_fwd_vort": (1 + st) * S}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--model", choices=["com", "coh", "csh", "css"], default="com")
    ap.add_argument("--grid", type=int, default=1024)
    ap.add_argument("--fp32", action="store_true")
    ap.add_argument("--stepper", choices=["rk4", "ab2"], default=None)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    a = ap.parse_args(argv)
    N = a.grid
    model = {"com": MODEL_COM, "coh": MODEL_COH, "csh": MODEL_CSH, "css": MODEL_CSS}[a.model]
    stepper = {"rk4": STEP_RK4, "ab2": STEP_AB2, None: STEP_RK4 if model == MODEL_COM else STEP_AB2}[a.stepper]
    prec = FP32 if a.fp32 else FP64
    if model == MODEL_COM:
        p = Params.make(Lx=2 * PI, Ly=2 * PI, pi=PI, dt=5e-5 * 1024 / N, mu=5e-4, eta=5e-4, CS=100.0,
                        spheat=5.0 / 3.0, ms=1.0, mu_0=1.0, kf=1.0, A=0.0, fix_curlB=0)
    elif model == MODEL_COH:
        p = Params.make(Lx=2 * PI, Ly=2 * PI, pi=PI, mux=1e-3, muy=1e-3, ms=1.0, CS=3.77, dt=1e-4 * 128 / N)
    elif model == MODEL_CSH:
        p = Params.make(pi=VPI, Lx=2 * VPI, Ly=2 * VPI, nu=1e-3, dt=1e-3 * 128 / N)
    else:
        p = Params.make(pi=VPI, Lx=2 * PI, Ly=2 * PI, nu=1e-3, alpha=1.0, dt=1e-3 * 128 / N, **{"lambda": 10.0})
    with Session(model, N, N, p, precision=prec) as s:
        if model == MODEL_COM:
            s.set_state_random(IC_ORSZAG_TANG, 0, e1=1e-3, e2=1e-3, kmin=8.0, kmax=16.0)
        elif model == MODEL_COH:
            s.set_state_random(IC_RANDOM_PHASE, 0, k0=4.0, e1=0.5, e2=0.01)
        else:
            s.set_state(initial.vorticity_random_phase(N, N, seed=0))
        s.step(stepper, a.warmup)
        ms = s.time_steps(stepper, a.steps)
        prof, total = s.profile_steps(stepper, a.steps)
    S = N * (N // 2 + 1) * (8 if a.fp32 else 16)
    table = kernel_bytes(model, stepper, S)
    kernels = {}
    for k, (t, n) in prof.items():
        per = t / n
        b = table.get(k, 0.0)
        kernels[k] = {"launches": n, "ms_per_launch": per, "share": t / total if total else None,
                      "alg_bytes_per_launch": b, "alg_GBps": b / (per / 1e3) / 1e9 if b else None}
    print(json.dumps({"model": a.model, "grid": N, "precision": "fp32" if a.fp32 else "fp64",
                      "stepper": "rk4" if stepper == STEP_RK4 else "ab2", "steps": a.steps,
                      "steps_per_s": a.steps / (ms / 1e3), "S_bytes": S, "kernels": kernels}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
