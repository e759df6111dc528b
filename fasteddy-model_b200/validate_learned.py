"""A-posteriori check of the learned SGS closure against a 2x-finer run of the plain model.

    python fasteddy-model_b200/validate_learned.py [--coarse NX NY NZ] [--spinup S] [--collect S]
                                                   [--eval S] [--sample S] [--train-steps N]

Dry convective boundary layer (the cbl_dry case): a fine run (2Nx x 2Ny x 2Nz, dx = 10 m,
dz = 5 m, dt = 0.0125 s) spins up, then its coarse-grained fields (2x2x2 Favre box filter,
fe_coarsen) are collected as training data for the network (inputs from the coarse grid,
targets the subfilter stresses and heat fluxes). From the coarse-grained fine state at the end
of the collection, three runs advance the same model time:

  fine      the plain model on the fine grid (coarse-grained for the comparison)
  learned   the coarse grid (dx = 20 m, dz = 10 m, dt = 0.025 s) with the network's stresses
  tke       the coarse grid with the TKE closure

and over the last part of that window the horizontally averaged profiles of resolved TKE,
0.5 <u'^2 + v'^2 + w'^2>, and of the total vertical heat flux, <w'theta'> plus the SGS flux
(tauTH3/rho; for the fine run the subfilter flux of the filter, which contains the fine run's
own SGS flux), are averaged in time. Reported: the relative L2 difference of each coarse run's
profiles from the fine run's over the lowest 80 % of the domain, and the time each run takes per
simulated second (CUDA events around a synchronous advance). One JSON line on stdout.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _load():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    return importlib.import_module("fasteddy-model_b200")


def _interior(a: np.ndarray, h: int = 3) -> np.ndarray:
    return a[..., h:-h, h:-h, h:-h]


def profiles(state: dict, sgs_heat: np.ndarray | None) -> tuple[np.ndarray, np.ndarray]:
    """Resolved TKE and total vertical heat flux per level from a state (flux form, halo 3) and
    the SGS heat flux tauTH3/rho of its interior cells (rows i, j, k with k fastest)."""
    f = _interior(state["hydroFlds"]).astype(np.float64)
    rho = f[0]
    u, v, w, th = f[1] / rho, f[2] / rho, f[3] / rho, f[4] / rho

    def dev(a):
        return a - a.mean(axis=(0, 1), keepdims=True)

    tke = 0.5 * (dev(u) ** 2 + dev(v) ** 2 + dev(w) ** 2).mean(axis=(0, 1))
    heat = (dev(w) * dev(th)).mean(axis=(0, 1))
    if sgs_heat is not None:
        heat = heat + sgs_heat.reshape(rho.shape).mean(axis=(0, 1))
    return tke, heat


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--coarse", type=int, nargs=3, default=(64, 64, 64), metavar=("NX", "NY", "NZ"))
    ap.add_argument("--spinup", type=float, default=600.0, help="model seconds of the fine spin-up")
    ap.add_argument("--collect", type=float, default=300.0, help="model seconds over which training data are taken")
    ap.add_argument("--eval", type=float, default=300.0, help="model seconds of the comparison window")
    ap.add_argument("--sample", type=float, default=30.0, help="model seconds between snapshots")
    ap.add_argument("--average", type=float, default=180.0, help="model seconds at the end of the window averaged")
    ap.add_argument("--train-steps", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=99)
    args = ap.parse_args(argv)

    fe = _load()
    import torch

    nx, ny, nz = args.coarse
    dtc, dtf = 0.025, 0.0125
    hf = fe.cases.setup_host("cbl_dry", 2 * nx, 2 * ny, 2 * nz, dx=10.0, dz=5.0, dt=dtf, seed=args.seed)
    fin, fcfg = hf.inputs(), hf.config()
    hf.cleanup()
    hc = fe.cases.setup_host("cbl_dry", nx, ny, nz, dx=20.0, dz=10.0, dt=dtc, seed=args.seed)
    cin, ccfg = hc.inputs(), hc.config()
    hc.cleanup()

    def coarse_domain():
        d = fe.Domain(ccfg)
        d.set_inputs(cin)
        return d

    fine = fe.Domain(fcfg)
    fine.set_inputs(fin)
    fine.autotune()
    probe = coarse_domain()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed_advance(d, steps):
        torch.cuda.synchronize()
        ev[0].record()
        d.advance(steps)
        ev[1].record()
        ev[1].synchronize()
        return ev[0].elapsed_time(ev[1])

    per_sample_f = int(round(args.sample / dtf))
    # spin-up and training data
    fine.advance(int(round(args.spinup / dtf)))
    Xs, Ts = [], []
    for _ in range(max(1, int(round(args.collect / args.sample)))):
        fine.advance(per_sample_f)
        tgt = fine.coarsen_into(probe)
        Xs.append(probe.sgs_sample()["X"])
        Ts.append(tgt)
    nsamples = int(sum(x.shape[0] for x in Xs))
    m = fe.Mlp(seed=args.seed)
    m.set_data(np.concatenate(Xs), np.concatenate(Ts))
    t0 = time.time()
    hist = m.train(args.train_steps, 8192, 2e-3)
    train_s = time.time() - t0
    del Xs, Ts

    # the three runs from the same coarse-grained state
    learned, tke = coarse_domain(), coarse_domain()
    fine.coarsen_into(learned)
    fine.coarsen_into(tke)
    learned.set_sgs_mlp(m)
    learned.autotune()
    tke.autotune()
    nsamp = max(1, int(round(args.eval / args.sample)))
    navg = max(1, int(round(args.average / args.sample)))
    acc = {k: [np.zeros(nz), np.zeros(nz)] for k in ("fine", "learned", "tke")}
    ms = {"fine": 0.0, "learned": 0.0, "tke": 0.0}
    finite = True
    for s in range(nsamp):
        ms["fine"] += timed_advance(fine, per_sample_f)
        ms["learned"] += timed_advance(learned, int(round(args.sample / dtc)))
        ms["tke"] += timed_advance(tke, int(round(args.sample / dtc)))
        if s >= nsamp - navg:
            tgt = fine.coarsen_into(probe)
            pf = profiles(probe.get_state(), tgt[:, 8])
            for name, d in (("learned", learned), ("tke", tke)):
                smp = d.sgs_sample()
                p = profiles(d.get_state(), smp["tau"][:, 8] / smp["rho"])
                finite = finite and bool(np.isfinite(p[0]).all() and np.isfinite(p[1]).all())
                acc[name][0] += p[0] / navg
                acc[name][1] += p[1] / navg
            acc["fine"][0] += pf[0] / navg
            acc["fine"][1] += pf[1] / navg
    top = int(0.8 * nz)
    out = {
        "case": "dry CBL, coarse %dx%dx%d (dx 20 m, dz 10 m), fine 2x in every direction" % (nx, ny, nz),
        "model_seconds": {"spinup": args.spinup, "collect": args.collect, "eval": args.eval, "averaged": args.average},
        "training": {"samples": nsamples, "steps": args.train_steps,
                     "loss_first": float(hist[0]), "loss_last": float(hist[-1]), "seconds": train_s},
        "profile_rel_l2_vs_fine": {
            name: {"resolved_tke": rel_l2(acc[name][0][:top], acc["fine"][0][:top]),
                   "heat_flux": rel_l2(acc[name][1][:top], acc["fine"][1][:top])}
            for name in ("learned", "tke")},
        "device_ms_per_model_second": {k: v / args.eval for k, v in ms.items()},
        "finite": finite,
        "profiles": {k: {"resolved_tke": acc[k][0].tolist(), "heat_flux": acc[k][1].tolist()} for k in acc},
    }
    for d in (fine, probe, learned, tke):
        d.close()
    m.close()
    return out


if __name__ == "__main__":
    print(json.dumps(main()))
