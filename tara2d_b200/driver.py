"""Time loop with the reference drivers' output files, everything computed on
the device.

    run(session, stepper, nsteps, every, outdir, snapshot_every=0, t0=0.0)

writes under `outdir`:
  * Energy.dat: one list-directed record per `every` steps (and one for the
    initial state): time, then the Energy.dat values of the model
    (MHD: Energy, B_Field, C2, C3, div_B_Tot as src/main2com.f95:616;
    hydro: Energy/2, y_Energy/2, C0, C1, C2, C3 as src/main2coh.f95:427-428);
  * Cross_Helicity.dat (MHD): time, <u.B>;
  * Energy_Spectra.dat: time, k, E(k) for every shell, per record;
  * fort.NNNNNNNN grid files every `snapshot_every` steps (0: none), named
    t + 100000 (MHD, src/main2com.f95:605) or t + 100 (hydro,
    src/main2coh.f95:415), t the step count.
The loop runs an explicit step count (the reference's REAL loop variable,
src/main2com.f95:352, makes its trip count depend on rounding).
"""
from __future__ import annotations

import os

from . import MODEL_COM, format_list_directed


def _values(model, vals):
    return list(vals[:5]) if model == MODEL_COM else list(vals[:6])


def run(session, stepper: int, nsteps: int, every: int, outdir: str, snapshot_every: int = 0, t0: float = 0.0):
    if every < 1 or nsteps < 0:
        raise ValueError("every >= 1 and nsteps >= 0")
    os.makedirs(outdir, exist_ok=True)
    model = session.model
    dt = session.params.dt
    base = 100000 if model == MODEL_COM else 100
    records = []
    with open(os.path.join(outdir, "Energy.dat"), "w") as fe, \
            open(os.path.join(outdir, "Energy_Spectra.dat"), "w") as fs, \
            open(os.path.join(outdir, "Cross_Helicity.dat") if model == MODEL_COM else os.devnull, "w") as fh:

        def record(t):
            vals, ek = session.diagnostics()
            time = t0 + t * dt
            fe.write(format_list_directed([time] + _values(model, vals)) + "\n")
            if model == MODEL_COM:
                fh.write(format_list_directed([time, vals[5]]) + "\n")
            for k, e in enumerate(ek):
                fs.write(format_list_directed([time, float(k), e]) + "\n")
            records.append((time, vals, ek))

        def snapshot(t):
            if snapshot_every and t % snapshot_every == 0:
                session.write_snapshot(os.path.join(outdir, "fort.%08d" % (t + base)))

        t = 0
        record(t)
        snapshot(t)
        while t < nsteps:
            n = min(every, nsteps - t)
            if snapshot_every:
                n = min(n, snapshot_every - t % snapshot_every)
            session.step(stepper, n)
            t += n
            if t % every == 0 or t == nsteps:
                record(t)
            snapshot(t)
    return records
