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


def test_roofline_traffic_is_read_from_the_committed_summary():
    t = bench.sweep_traffic()
    assert t is not None and 1e6 < t < 1e9
    with open(os.path.join(bench.ROOT, "profiles", "k_sweep_sheet256_fold.md")) as f:
        assert any(line.startswith("traffic_bytes_per_launch: %d" % int(t)) for line in f)


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
            return x, v, t + st.dt, {"iterations": 7}

    monkeypatch.setattr(oracle, "Solver", FakeSolver)
    sc = bench.workload()
    state = (sc.x0, sc.v0, 0.0)
    done, dt, its, warm = bench.cpu_reference_run(sc, state, 2, 60.0, 3, warmup=1)
    assert done == 2 and warm == 1 and its == [7, 7] and dt >= 0.0
    assert seen == [(0, 0.0, bench.TOLERANCE, bench.ITERATION_CAP, 3)] * 3
