"""TimeStepLength (src/dynamics.f90:511-600) and the failure paths of a step.

* The CFL number reported with a constant time step equals the oracle's
  U_dx_max * dt (enable_CFL_check).
* Variable time steps: each step's length is min(CFL / U_dx_max, dt_max)
  of the state at its start, shortened so as not to pass end_time; the GPU
  state, the length of the last step and the time follow the oracle (FP64
  1e-12), and the mixed path follows within its tolerance.
* A bounded device-side wait that runs out (a plane whose copies the
  kernels do not issue, elmm_set_fault_injection) makes elmm_step return
  ELMM_ERR_TIMEOUT instead of hanging; the same handle then steps normally
  and matches a fresh one bit for bit.

The oracle's variable step is checked on the CPU against the formula
evaluated with numpy on the state."""
import numpy as np
import pytest

from conftest import rel
from gpu_elmm_b200.config import grid_of, make_config
from gpu_elmm_b200.workloads import interiors, log_profile_state
from oracle import Oracle


def _u_dx_max(g, U, V, W, dx=1.0, dy=1.0, dz=1.0):
    o = 2
    nx, ny, nz = g.Prnx, g.Prny, g.Prnz
    u = np.abs(U[o + 1:o + nz + 1, o + 1:o + ny + 1, o:o + nx + 1])
    v = np.abs(V[o + 1:o + nz + 1, o:o + ny + 1, o + 1:o + nx + 1])
    w = np.abs(W[o:o + nz + 1, o + 1:o + ny + 1, o + 1:o + nx + 1])
    p = np.maximum(u[:, :, 1:], u[:, :, :-1]) / dx + np.maximum(v[:, 1:, :], v[:, :-1, :]) / dy + \
        np.maximum(w[1:], w[:-1]) / dz
    return float(p.max())


def test_oracle_variable_step_length():
    cfg = make_config(32, 24, 16, variable_dt=True, cfl=0.4, dt_max=0.05, end_time=0.3)
    g = grid_of(cfg)
    o = Oracle(cfg)
    o.set_state(*log_profile_state(g, seed=2))
    o.project(1.0)
    t = 0.0
    for _ in range(6):
        o.bound()
        U, V, W, _ = o.state()
        expect = min(0.4 / _u_dx_max(g, U, V, W), 0.05)
        expect = min(expect, 0.3 - t)
        o.step(1)
        t2, dt = o.clock()
        assert dt == pytest.approx(expect, rel=1e-14) and t2 == pytest.approx(t + dt, rel=1e-14)
        t = t2
    assert t <= 0.3 + 1e-15


@pytest.mark.gpu
def test_reported_cfl_follows_the_oracle():
    from gpu_elmm_b200 import lib as L
    cfg = make_config(48, 32, 24, cfl_check=1)
    g = grid_of(cfg)
    o = Oracle(cfg)
    o.set_state(*log_profile_state(g, seed=3))
    o.project(1.0)
    d = L.Domain(cfg)
    d.upload(*o.state())
    for _ in range(3):
        _, cfl_o = o.step(1)
        s = d.step(1)
        assert cfl_o > 0 and s.cfl == pytest.approx(cfl_o, rel=1e-13), (s.cfl, cfl_o)
    d.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_variable_time_steps_follow_the_oracle(precision):
    from gpu_elmm_b200 import lib as L
    kw = dict(variable_dt=True, cfl=0.35, dt_max=0.1)  # the CFL limit (~0.04) sets the length
    cfg = make_config(48, 32, 24, precision=precision, **kw)
    g = grid_of(cfg)
    o = Oracle(make_config(48, 32, 24, **kw))
    o.set_state(*log_profile_state(g, seed=4))
    o.project(1.0)
    d = L.Domain(cfg)
    d.upload(*o.state())
    tol = 1e-13 if precision == 0 else 1e-5
    dts = []
    for n in (1, 3, 6):
        o.step(n)
        s = d.step(n)
        t_o, dt_o = o.clock()
        dts.append(dt_o)
        assert s.dt == pytest.approx(dt_o, rel=tol) and s.time == pytest.approx(t_o, rel=tol), (s.dt, dt_o, s.time, t_o)
        e = [rel(a, b) for a, b in zip(interiors(g, *d.download()), interiors(g, *o.state()))]
        if precision == 0:
            assert max(e[:3]) < 1e-12 and e[3] < 1e-11, e
        else:
            assert max(e[:3]) < 1e-5, e
    assert len(set(round(x, 15) for x in dts)) > 1  # the length varies
    d.close()


@pytest.mark.gpu
def test_variable_time_steps_stop_at_end_time():
    """The step that would pass end_time ends there (as the oracle's); a step
    started at end_time is reported."""
    from gpu_elmm_b200 import lib as L
    kw = dict(variable_dt=True, cfl=0.35, dt_max=0.1, end_time=0.1)
    cfg = make_config(32, 24, 16, **kw)
    g = grid_of(cfg)
    o = Oracle(cfg)
    o.set_state(*log_profile_state(g, seed=8))
    o.project(1.0)
    d = L.Domain(cfg)
    d.upload(*o.state())
    for _ in range(20):
        o.step(1)
        s = d.step(1)
        t_o, dt_o = o.clock()
        assert s.dt == pytest.approx(dt_o, rel=1e-13) and s.time == pytest.approx(t_o, rel=1e-13)
        if s.time >= 0.1 - 1e-12:
            break
    assert s.time == pytest.approx(0.1, rel=1e-13)
    e = [rel(a, b) for a, b in zip(interiors(g, *d.download()), interiors(g, *o.state()))]
    assert max(e[:3]) < 1e-12, e
    with pytest.raises(L.ElmmError) as err:
        d.step(1)
    assert err.value.code == 6
    d.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_a_wait_that_runs_out_is_reported_and_the_handle_recovers(precision):
    from gpu_elmm_b200 import lib as L
    cfg = make_config(64, 32, 24, precision=precision)
    g = grid_of(cfg)
    st = log_profile_state(g, seed=5)
    d, ref = L.Domain(cfg), L.Domain(cfg)
    for x in (d, ref):
        x.upload(*st)
        x.project(1.0)
    s0 = d.download()
    d.set_fault_injection(wait_limit=256, skip_plane=5)
    with pytest.raises(L.ElmmError) as e:
        d.step(1)
    assert e.value.code == 5, str(e.value)
    d.set_fault_injection()  # back to normal operation
    d.upload(*s0)
    ref.upload(*ref.download())  # the same upload (the mixed path's offsets come from the uploaded state)
    d.step(2)
    ref.step(2)
    for a, b in zip(d.download(), ref.download()):
        assert np.array_equal(a, b)
    d.close()
    ref.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_variable_time_steps_in_a_batch_equal_the_runs_alone(precision):
    """Each domain of a batch takes its own variable step (k_dt works per
    domain): two domains of different sizes, targets and starting states,
    stepped together, equal the same domains stepped alone, bit for bit."""
    from gpu_elmm_b200 import lib as L
    kws = [dict(variable_dt=True, cfl=0.35, dt_max=0.1), dict(variable_dt=True, cfl=0.2, dt_max=0.05)]
    sizes = [(48, 32, 24), (32, 32, 16)]
    cfgs = [make_config(*n, precision=precision, **kw) for n, kw in zip(sizes, kws)]
    states = [log_profile_state(grid_of(c), seed=20 + q) for q, c in enumerate(cfgs)]
    b = L.Batch(cfgs)
    for q, st in enumerate(states):
        b.upload(q, *st)
    b.project(1.0)
    b.step(4)
    for q, (c, st) in enumerate(zip(cfgs, states)):
        d = L.Domain(c)
        d.upload(*st)
        d.project(1.0)
        d.set_tuning(**b.tuning())
        s = d.step(4)
        assert s.dt > 0
        for x, y in zip(b.download(q), d.download()):
            assert np.array_equal(x, y), q
        d.close()
    b.close()
