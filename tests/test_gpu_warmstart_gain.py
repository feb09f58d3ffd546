"""What the trained network gains over the method without it.

A residual surrogate (the physics start plus a learned correction, see
ekpnp.warmstart) is trained on the GPU, by the project's own tensor-core
kernels, on steady states that the batched solver produced for channels
drawn from a slice of the batched workload's distributions (16 columns,
32-80 rows, kappa*H 2-20, zeta -3 to -1, E_x 1e-5 to 1e-3, D 0.04-0.08,
seed 3).  32 held-out channels of the same slice (seed 4) then run to the
steady-state residual < 1e-8 from three starts:
  * the network's start (with the cold-start fallback for a channel whose
    residual rises),
  * the physics start without the network: Newton Poisson-Boltzmann ions and
    potential and the electro-osmotic velocity u_HS (1 - psi/zeta),
  * the uniform cold start.
Every channel must reach steady state from the network's start, in fewer
summed steps and less wall time than from either start without the network.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SLICE = dict(nx_choices=(16,), ny_range=(32, 80), kappa_h_range=(2.0, 20.0), zeta_range=(-3.0, -1.0),
             ex_range=(1e-5, 1e-3), diff_range=(0.04, 0.08))
CAP = 100_000


@pytest.fixture(scope="module")
def runs():
    import ekpnp
    from ekpnp import warmstart as ws
    ekpnp.set_device(0)
    train = ekpnp.batch_specs(768, seed=3, **SLICE)
    T, conv, _ = ws.generate_steady_states(train, nx=16, max_steps=CAP, check=1000)
    ok = conv & np.all(np.isfinite(T), axis=1)
    assert ok.sum() >= 600, int(ok.sum())
    sg = ws.Surrogate("residual", seed=7)
    try:
        sg.fit([s for s, o in zip(train, ok) if o], T[ok], iters=4000, lr=2e-3)
        evals = ekpnp.batch_specs(32, seed=4, **SLICE)
        kw = dict(max_steps=CAP, check=1000)
        out = {"network": ws.warm_start_run(sg, evals, **kw),
               "physics": ws.physics_start_run(evals, **kw),
               "cold": ws.cold_start_run(evals, **kw)}
    finally:
        sg.close()
    summary = {k: dict(wall_s=round(r["wall_s"], 3), converged=int(np.sum(r["steps"] >= 0)),
                       sum_steps=int(np.where(r["steps"] >= 0, r["steps"], CAP).sum()),
                       median_steps=float(np.median(np.where(r["steps"] >= 0, r["steps"], CAP))))
               for k, r in out.items()}
    print("time to residual < 1e-8, 32 held-out channels:", summary)
    return out, summary


def test_network_start_reaches_steady_state(runs):
    out, summary = runs
    assert summary["network"]["converged"] == 32, summary
    assert len(out["network"]["fallback"]) <= 2, summary


def test_network_start_beats_the_starts_without_it(runs):
    _, summary = runs
    net, phys, cold = summary["network"], summary["physics"], summary["cold"]
    assert net["sum_steps"] < phys["sum_steps"] < cold["sum_steps"], summary
    assert net["wall_s"] < phys["wall_s"] and net["wall_s"] < cold["wall_s"], summary
