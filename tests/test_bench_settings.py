"""bench.py's settings contract, on the CPU: the equal-residual legs carry the
residual target, stall refresh and acceleration; the fixed-iteration legs and
the CPU reference arm run the reference's iteration (no target, no
acceleration); the roofline traffic comes from the committed ncu summary."""
import os

import bench


def test_equal_residual_settings():
    sc = bench.workload()
    st = bench.step_settings(sc, 1)
    assert st.iterations == bench.ITERATION_CAP and st.init_mode == 1
    assert st.residual_tolerance == bench.TOLERANCE and st.residual_check_every == bench.CHECK_EVERY
    assert st.stall_refresh == bench.STALL_REFRESH and st.acceleration == bench.ACCELERATION
    plain = bench.step_settings(sc, 0, acceleration=0.0)
    assert plain.init_mode == 0 and plain.acceleration == 0.0 and plain.residual_tolerance == bench.TOLERANCE


def test_fixed_iteration_settings_are_the_reference_step():
    sc = bench.workload()
    st = bench.step_settings(sc, 0, bench.FIXED_ITERATIONS)
    assert st.iterations == bench.FIXED_ITERATIONS
    assert st.residual_tolerance == 0.0 and st.residual_check_every == 0
    assert st.stall_refresh == 0 and st.acceleration == 0.0 and st.init_mode == 0


def test_config_names_the_workload_and_its_target():
    sc = bench.workload()
    c = bench.config_dict(sc, 1)
    assert c["vertices"] == 65536 and c["triangles"] == 130050
    assert c["residual_tolerance"] == bench.TOLERANCE and "fold" in c["workload"]
    assert "flushed" in c["l2"]


def test_roofline_traffic_is_a_recorded_constant():
    """The sweep's DRAM bytes per launch are a constant recorded beside the ncu
    command that measured them; bench.py reads no file for them."""
    t = bench.SWEEP_TRAFFIC_BYTES
    assert 1e6 < t < 1e9
    src = open(os.path.join(bench.ROOT, "bench.py")).read()
    assert "profiles/" not in src and "ncu --set full --clock-control none -k regex:k_sweep" in src


def test_cpu_reference_arm_runs_the_reference_iteration(monkeypatch):
    """The reference arm steps the oracle with the adaptive init and neither
    acceleration nor the learned guess, at the same residual target."""
    import oracle

    seen = []

    class FakeSolver:
        def __init__(self, scene, threads=1):
            self.threads = threads

        def step(self, x, v, t, st):
            seen.append((st.init_mode, st.acceleration, st.residual_tolerance, st.iterations, self.threads))
            return x, v, t + st.dt, {"iterations": 7, "relative_force_residual": 1e-3}

    monkeypatch.setattr(oracle, "Solver", FakeSolver)
    sc = bench.workload()
    state = (sc.x0, sc.v0, 0.0)
    done, dt, (its, force), warm = bench.cpu_reference_run(sc, state, 2, 60.0, 3, warmup=1)
    assert done == 2 and warm == 1 and its == [7, 7] and force == [1e-3, 1e-3] and dt >= 0.0
    assert seen == [(0, 0.0, bench.TOLERANCE, bench.ITERATION_CAP, 3)] * 3


def test_cpu_reference_arm_runs_every_timed_step_within_its_budget(monkeypatch):
    """The reference arm times all K steps unless they outlast the budget;
    the warm-up has a budget of its own."""
    import oracle

    class FakeSolver:
        def __init__(self, scene, threads=1):
            pass

        def step(self, x, v, t, st):
            return x, v, t + st.dt, {"iterations": 3, "relative_force_residual": 1e-3}

    monkeypatch.setattr(oracle, "Solver", FakeSolver)
    sc = bench.workload()
    done, _, (its, _), warm = bench.cpu_reference_run(sc, (sc.x0, sc.v0, 0.0), 20, 1e6, 1, warmup=5,
                                                      warmup_budget_s=1e6)
    assert done == 20 and warm == 5 and len(its) == 20
