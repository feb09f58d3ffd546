"""Learned warm start of batched channels (new; the reference starts every
run from its Poisson-Boltzmann initialisation, LBM.cu:95-145, or a file).

Pipeline:
  1. steady states   the batched solver runs many channels (drawn from the
                     batched workload's distributions) to a steady state,
                     residual < tol; the cross-channel profiles of psi, c+, c-
                     and u_x (row means; walls uniform along x) are encoded as
                     four 128-point profiles on Chebyshev-Lobatto points of
                     s = y / (ny - 1), which cluster at the walls where the
                     double layers are.
  2. training        the MLP (ekpnp.mlp: tcgen05 GEMMs, Adam) maps the four
                     normalised descriptors (kappa*H, zeta, E_x, N_y) to those
                     512 numbers.
  3. warm start      a channel's fields are decoded from the network's output
                     and the solver iterates from them to the same residual.
                     The solver judges the start: a channel whose residual
                     rises between two checks early on, or goes non-finite, is
                     re-run from the uniform cold start.
  x-reduced start    (xreduced_start_run) the relaxation itself runs on 16
                     columns, from the network's or the cold start, and the
                     relaxed state is tiled along x into the full channel.
Profile encoding (all O(1)): psi / zeta, ln(c+/c0) / (-zeta), ln(c-/c0) / zeta,
u_x / u_HS with u_HS = -eps zeta E_x / (rho0 nu) the Helmholtz-Smoluchowski
speed (Boltzmann equilibrium and the electro-osmotic profile make the four
nearly 1 - s-shaped curves of one double layer).
"""
from __future__ import annotations

import time

import numpy as np

from ._lib import STORE_F32
from .batch import Batch
from .params import spec_params

NS = 128
S = 0.5 * (1.0 - np.cos(np.pi * np.arange(NS) / (NS - 1)))  # Chebyshev-Lobatto points on [0, 1]
RANGES = {"kappa_h": (1.0, 50.0), "zeta": (-4.0, -0.5), "ex": (1e-5, 1e-3), "ny": (32, 512)}


def _lin(v, lo, hi):
    return 2.0 * (v - lo) / (hi - lo) - 1.0


def features(specs):
    """(n, 4) float32: log kappa*H, zeta, log E_x, log N_y mapped to [-1, 1]."""
    out = np.empty((len(specs), 4), dtype=np.float32)
    for i, s in enumerate(specs):
        out[i, 0] = _lin(np.log(s["kappa_h"]), *np.log(RANGES["kappa_h"]))
        out[i, 1] = _lin(s["zeta"], *RANGES["zeta"])
        out[i, 2] = _lin(np.log(s["ex"]), *np.log(RANGES["ex"]))
        out[i, 3] = _lin(np.log(s["ny"]), *np.log(RANGES["ny"]))
    return out


def u_hs(p):
    return -p["eps"] * p["zeta_lo"] * p["ext_x"] / (p["rho0"] * p["nu"])


def encode(spec, prof):
    """512 float32 targets from 1-D profiles (ny values each) of psi, cp, cn, ux."""
    p = spec_params(spec, 0)
    ny, z = spec["ny"], spec["zeta"]
    y = S * (ny - 1)
    grid = np.arange(ny)
    cols = (prof["psi"] / z,
            np.log(np.maximum(prof["cp"], 1e-300) / p["c0"]) / (-z),
            np.log(np.maximum(prof["cn"], 1e-300) / p["c0"]) / z,
            prof["ux"] / u_hs(p))
    return np.concatenate([np.interp(y, grid, c) for c in cols]).astype(np.float32)


def decode(spec, vec, nx=None):
    """Fields (ny x nx) of a channel from 512 network outputs."""
    p = spec_params(spec, 0)
    nx = spec["nx"] if nx is None else nx
    ny, z = spec["ny"], spec["zeta"]
    t = np.asarray(vec, dtype=np.float64).reshape(4, NS)
    s = np.arange(ny) / (ny - 1)
    psi = z * np.interp(s, S, t[0])
    psi[0] = psi[-1] = z
    cp = p["c0"] * np.exp(-z * np.interp(s, S, t[1]))
    cn = p["c0"] * np.exp(z * np.interp(s, S, t[2]))
    ux = u_hs(p) * np.interp(s, S, t[3])
    ux[0] = ux[-1] = 0.0
    col = lambda v: np.repeat(v[:, None], nx, axis=1)
    return dict(rho=np.full((ny, nx), p["rho0"]), ux=col(ux), uy=np.zeros((ny, nx)), cp=col(cp), cn=col(cn),
                psi=col(psi))


def profiles(ch):
    """Row means of psi, cp, cn, ux of a channel."""
    f = ch.get_fields(("psi", "cp", "cn", "ux"))
    return {k: v.mean(axis=1) for k, v in f.items()}


def cold_state(spec, nx=None):
    p = spec_params(spec, 0)
    nx = spec["nx"] if nx is None else nx
    ny = spec["ny"]
    z = np.zeros((ny, nx))
    return dict(rho=np.full((ny, nx), p["rho0"]), ux=z, uy=z.copy(), cp=np.full((ny, nx), p["c0"]),
                cn=np.full((ny, nx), p["c0"]), psi=z.copy())


def pb_column(spec):
    """Discrete 1-D Poisson-Boltzmann potential across the channel (the
    equation of ek_init_poisson_boltzmann's Newton form):
        (psi[j-1] - 2 psi[j] + psi[j+1]) / dy^2 + g (exp(-psi[j]) - exp(psi[j])) = 0,
    psi = zeta on both walls, g = f_charge c0 / eps; damped Newton (each
    update changes psi by at most 1) from the linear profile."""
    from scipy.linalg import solve_banded
    p = spec_params(spec, 0)
    ny, z = spec["ny"], spec["zeta"]
    g = p["f_charge"] * p["c0"] / p["eps"]
    inv = 1.0 / (p["dy"] * p["dy"])
    psi = np.full(ny, float(z))
    ab = np.zeros((3, ny - 2))
    polish = -1
    for _ in range(500):
        v = psi[1:-1]
        em, ep = np.exp(-v), np.exp(v)
        G = (psi[:-2] - 2.0 * v + psi[2:]) * inv + g * (em - ep)
        ab[0, 1:] = inv
        ab[1] = -2.0 * inv - g * (em + ep)
        ab[2, :-1] = inv
        d = solve_banded((1, 1), ab, -G)
        m = float(np.abs(d).max())
        damp = 1.0 / m if m > 1.0 else 1.0
        psi[1:-1] += damp * d
        if polish < 0 and damp == 1.0 and m < 1e-9 * max(abs(z), 1.0):
            polish = 2
        if polish >= 0:
            polish -= 1
            if polish < 0:
                return psi
    raise RuntimeError("Poisson-Boltzmann Newton iteration did not converge")


def physics_profiles(spec):
    """Poisson-Boltzmann ions and potential, and the electro-osmotic velocity
    u = u_HS (1 - psi/zeta) of that potential (1-D profiles)."""
    p = spec_params(spec, 0)
    psi = pb_column(spec)
    return dict(psi=psi, cp=p["c0"] * np.exp(-psi), cn=p["c0"] * np.exp(psi),
                ux=u_hs(p) * (1.0 - psi / spec["zeta"]))


def profile_fields(spec, prof, nx=None):
    p = spec_params(spec, 0)
    nx = spec["nx"] if nx is None else nx
    ny = spec["ny"]
    col = lambda v: np.repeat(np.asarray(v, dtype=np.float64)[:, None], nx, axis=1)
    return dict(rho=np.full((ny, nx), p["rho0"]), ux=col(prof["ux"]), uy=np.zeros((ny, nx)), cp=col(prof["cp"]),
                cn=col(prof["cn"]), psi=col(prof["psi"]))


def physics_start(batch, specs):
    for ch, s in zip(batch, specs):
        ch.set_fields(**profile_fields(s, physics_profiles(s), nx=ch.nx))


# Residual recorded for a channel at the check where it is restarted and the
# one after (finite: the channel is neither converged nor diverged there).
UNJUDGED = 1e300


def run_to_steady(batch, tol=1e-8, check=1000, max_steps=200_000, judge=None, freeze=True, restart=None):
    """Step the batch until every channel has residual < tol (checked every
    `check` steps, an even number) or diverged, or max_steps.  With freeze,
    channels stop stepping once converged or diverged (and, with judge, once
    judged), so the work shrinks as they finish.  Returns per-channel steps to
    steady (-1: not reached), a diverged mask, the residual history (one row
    per check; frozen channels repeat their last value), the wall time in
    seconds (host clock, checks included) and the node updates of the stepping
    channels (node_steps).  judge=(k1, k2): also return the channels whose
    worst residual rose from check k1 to check k2.  restart(indices): with
    judge, such channels (and those that go non-finite first) are handed to
    restart -- which gives them a new start in place (Batch.restart) -- once
    each, instead of being frozen; they step on with the others, their steps
    to steady count from the batch's start, and the check right after a
    restart (which compares with the state before it) is not judged."""
    n = len(batch)
    steps_to = np.full(n, -1, dtype=np.int64)
    hist = []
    done = np.zeros(n, bool)
    restarted = np.zeros(n, bool)
    fresh = np.zeros(n, bool)  # restarted at the previous check
    last = np.full(n, np.inf)
    node_steps = 0
    batch.sync()
    t0 = time.perf_counter()
    batch.residual(check)  # first snapshot
    while batch.steps < max_steps:
        k = min(check, max_steps - batch.steps)
        node_steps += batch.active[1] * k
        batch.step(k)
        r = batch.residual(check)[:, 4]
        r = np.where(fresh, UNJUDGED, r)
        fresh[:] = False
        r = np.where(done, last, r)
        if restart is not None and judge is not None:
            cand = ~restarted & ~done & ~np.isfinite(r)
            if len(hist) + 1 > judge[1]:
                cand |= ~restarted & ~done & rising_channels(np.array(hist + [r]), *judge)
            if cand.any():
                restart(np.nonzero(cand)[0])
                restarted |= cand
                fresh |= cand
                r = np.where(cand, UNJUDGED, r)
        last = r
        hist.append(r)
        ok = np.isfinite(r)
        newly = (steps_to < 0) & ok & (r < tol)
        steps_to[newly] = batch.steps
        if np.all((steps_to >= 0) | ~ok):
            break
        if freeze:
            stop = (steps_to >= 0) | ~ok
            if judge is not None and restart is None and len(hist) > judge[1]:
                stop |= rising_channels(np.array(hist), *judge)
            if np.any(stop & ~done):
                done |= stop
                batch.set_active(~done)
    wall = time.perf_counter() - t0
    hist = np.array(hist)
    diverged = ~np.isfinite(hist[-1]) if len(hist) else np.zeros(n, bool)
    if judge is None:
        rising = None
    elif restart is not None:
        rising = restarted
    else:
        rising = rising_channels(hist, *judge)
    return dict(steps=steps_to, diverged=diverged, history=hist, wall_s=wall, rising=rising, node_steps=node_steps,
                restarted=restarted)


def rising_channels(hist, k1, k2):
    """Channels whose residual at check k2 is above that at check k1, or that
    are non-finite at any check so far (hist: checks x channels)."""
    hist = np.asarray(hist, dtype=np.float64)
    n = hist.shape[1]
    bad = ~np.all(np.isfinite(hist), axis=0) if len(hist) else np.zeros(n, bool)
    if len(hist) > k2:
        with np.errstate(invalid="ignore"):
            bad |= hist[k2] > hist[k1]
    return bad


def generate_steady_states(specs, nx=16, tol=1e-8, check=1000, max_steps=50_000, storage=STORE_F32, cycle=200):
    """Targets (n x 512) of the channels described by specs, run from the
    physics start on nx columns (walls uniform along x: the steady state does
    not depend on x).  Returns (targets, converged mask, run info)."""
    specs = [dict(s, nx=nx) for s in specs]
    with Batch([spec_params(s, storage) for s in specs]) as b:
        physics_start(b, specs)
        b.set_cycle(cycle)
        b.init_equilibrium()
        info = run_to_steady(b, tol=tol, check=check, max_steps=max_steps)
        targets = np.stack([encode(s, profiles(ch)) for s, ch in zip(specs, b)])
    conv = (info["steps"] >= 0) & np.all(np.isfinite(targets), axis=1)
    return targets, conv, info


class Surrogate:
    """The warm-start network and its target encoding.

    mode "direct": the network's 512 outputs are the encoded profiles.
    mode "residual": they are the difference between the encoded steady
    profiles and the encoded physics start (Poisson-Boltzmann ions and
    potential, electro-osmotic velocity), scaled per output by its spread over
    the training set; the start is the physics profiles plus that learned
    correction of what the lattice's own steady state does differently."""

    def __init__(self, mode="direct", batch=256, seed=0):
        from .mlp import Mlp
        if mode not in ("direct", "residual"):
            raise ValueError("mode is 'direct' or 'residual'")
        self.mode = mode
        self.net = Mlp(batch=batch, seed=seed)
        self.offset = np.zeros(4 * NS, dtype=np.float32)
        self.scale = np.ones(4 * NS, dtype=np.float32)

    def close(self):
        self.net.close()

    def _base(self, specs):
        """Encoded physics start (zeros for "direct") and the per-channel factor
        of the velocity block: the physics start's peak u_x / u_HS, so that the
        velocity correction of a thick double layer (peak far below u_HS) is
        learned relative to its own size."""
        if self.mode == "direct":
            return np.zeros((len(specs), 4 * NS), dtype=np.float32), np.ones(len(specs), dtype=np.float32)
        base = np.stack([encode(s, physics_profiles(s)) for s in specs])
        peak = np.maximum(base[:, 3 * NS:].max(axis=1), 1e-3).astype(np.float32)
        return base, peak

    def _unscale(self, specs, y):
        base, peak = self._base(specs)
        y = y.copy()
        y[:, 3 * NS:] *= peak[:, None]
        return base + y

    def fit(self, specs, targets, iters=8000, lr=2e-3, chunks=8):
        """Adam with a cosine learning-rate decay in `chunks` steps; returns the
        per-iteration losses (of the scaled targets)."""
        base, peak = self._base(specs)
        y = targets - base
        y[:, 3 * NS:] /= peak[:, None]
        self.offset = y.mean(axis=0).astype(np.float32)
        self.scale = np.maximum(y.std(axis=0), 1e-6).astype(np.float32)
        self.net.set_data(features(specs), (y - self.offset) / self.scale)
        losses = []
        per = max(1, iters // chunks)
        for k in range(chunks):
            rate = lr * max(0.5 * (1.0 + np.cos(np.pi * k / chunks)), 0.02)
            losses.append(self.net.train(per, rate))
        return np.concatenate(losses)

    def predict(self, specs):
        return self._unscale(specs, self.net.forward(features(specs)) * self.scale + self.offset)

    def fields(self, specs):
        return [decode(s, v) for s, v in zip(specs, self.predict(specs))]


def start_run(specs, fields, tol=1e-8, check=1000, max_steps=200_000, storage=STORE_F32, cycle=200, judge=None):
    """Run the channels from the given start fields to steady state.  With
    judge=(k1, k2) the channels whose residual rises between checks k1 and k2,
    or that diverge, are restarted in place from the uniform cold start and
    step on with the others (their steps count from the batch's start; the
    wall time covers the whole batch)."""
    t0 = time.perf_counter()
    with Batch([spec_params(s, storage) for s in specs]) as b:
        for ch, f in zip(b, fields):
            ch.set_fields(**f)
        b.set_cycle(cycle)
        b.init_equilibrium()
        info = run_to_steady(b, tol=tol, check=check, max_steps=max_steps, judge=judge,
                             restart=None if judge is None else cold_restart(b, specs))
        final = [profiles(ch) for ch in b]
    fallback = np.nonzero(info["restarted"])[0]
    return dict(steps=info["steps"].copy(), wall_s=time.perf_counter() - t0, first=info, fallback=fallback,
                final=final, diverged=info["diverged"])


def cold_restart(batch, specs):
    """A restart callback for run_to_steady: the channels' uniform cold start,
    loaded and restarted in place."""
    def restart(idx):
        mask = np.zeros(len(batch), bool)
        for i in idx:
            batch[i].set_fields(**cold_state(specs[i]))
            mask[i] = True
        batch.restart(mask)
    return restart


def warm_start_run(surrogate, specs, judge=(1, 3), **kw):
    """Time to steady from the network's start with the cold-start fallback;
    the wall time includes inference and decoding."""
    t0 = time.perf_counter()
    fields = surrogate.fields(specs)
    out = start_run(specs, fields, judge=judge, **kw)
    out["wall_s"] = time.perf_counter() - t0
    out["fields"] = fields
    return out


def cold_start_run(specs, **kw):
    return start_run(specs, [cold_state(s) for s in specs], **kw)


def physics_start_run(specs, **kw):
    t0 = time.perf_counter()
    fields = [profile_fields(s, physics_profiles(s)) for s in specs]
    out = start_run(specs, fields, **kw)
    out["wall_s"] = time.perf_counter() - t0
    out["fields"] = fields
    return out


def xreduced_start_run(specs, start="cold", surrogate=None, narrow_nx=16, tol=1e-8, check=1000,
                       max_steps=200_000, narrow_max_steps=None, storage=STORE_F32, cycle=200, judge=(1, 3)):
    """Time to steady through an x-reduced relaxation.  Walls uniform along x
    make the steady state independent of x, so each channel first relaxes on
    narrow_nx columns (start "cold": the uniform cold start; "surrogate": the
    network's start, judged as in warm_start_run with the cold start as
    in-place fallback; "physics": the Poisson-Boltzmann/electro-osmotic start without
    the network), then its relaxed state is tiled along x into the full channel
    (ek_tile_x) and the full batch steps to the same residual.  Steps and wall
    time count both stages (inference, both batches' set-up and the copies
    included).  narrow_max_steps caps the narrow stage (default max_steps):
    its steps cost 16/nx of a full-width step's work."""
    t0 = time.perf_counter()
    nspecs = [dict(s, nx=narrow_nx) for s in specs]
    for s in specs:
        if s["nx"] % narrow_nx:
            raise ValueError("every nx must be a multiple of narrow_nx")
    if start == "surrogate":
        nfields = surrogate.fields(nspecs)
    elif start == "cold":
        nfields = [cold_state(s) for s in nspecs]
        judge = None
    elif start == "physics":
        nfields = [profile_fields(s, physics_profiles(s)) for s in nspecs]
        judge = None
    else:
        raise ValueError("start is 'cold', 'physics' or 'surrogate'")
    kw = dict(tol=tol, check=check, max_steps=max_steps)
    nkw = dict(kw, max_steps=max_steps if narrow_max_steps is None else narrow_max_steps)
    batches = []
    try:
        nb = Batch([spec_params(s, storage) for s in nspecs])
        batches.append(nb)
        for ch, f in zip(nb, nfields):
            ch.set_fields(**f)
        nb.set_cycle(cycle)
        nb.init_equilibrium()
        narrow = run_to_steady(nb, judge=judge, restart=None if judge is None else cold_restart(nb, nspecs), **nkw)
        src = list(nb)
        nsteps = narrow["steps"].copy()
        fallback = np.nonzero(narrow["restarted"])[0]
        t_narrow = time.perf_counter() - t0
        with Batch([spec_params(s, storage) for s in specs]) as wb:
            wb.set_cycle(cycle)
            wb.init_equilibrium()
            for w, n in zip(wb, src):
                w.tile_x(n)
            wb.resync()
            full = run_to_steady(wb, **kw)
            final = [profiles(ch) for ch in wb]
    finally:
        for b in batches:
            b.close()
    fsteps = full["steps"]
    steps = np.where((nsteps >= 0) & (fsteps >= 0), nsteps + fsteps, -1)
    return dict(steps=steps, narrow_steps=nsteps, full_steps=fsteps, wall_s=time.perf_counter() - t0,
                narrow_wall_s=t_narrow, fallback=fallback, final=final, diverged=full["diverged"],
                fields=nfields)


def surrogate_error(spec, fields, prof):
    """Max-abs error of the start against a converged profile, relative to the
    converged field's max-abs, per field."""
    out = {}
    for k in ("psi", "cp", "cn", "ux"):
        start = fields[k].mean(axis=1)
        out[k] = float(np.abs(start - prof[k]).max() / max(np.abs(prof[k]).max(), 1e-300))
    return out
