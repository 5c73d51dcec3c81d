"""Multi-member batch (tracer_batch_*): both persistent step paths (one
cooperative launch per step; one launch per phase and wave), with and
without their CUDA graphs, at any tile, and mixed step by step, give the bits
of the per-member separate launches, also after a member's velocity changes;
the bounded grid barrier reports a timeout instead of hanging; the autotuner
keeps the tracer state."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture()
def small_batch(api):
    from fesom2_tracer_dwarf_b200.batch import TracerBatch
    from fesom2_tracer_dwarf_b200.workloads import build_ensemble, ensemble_specs
    specs = ensemble_specs(3, seed=5, nx_range=(12, 30), nl_range=(6, 14))
    b = TracerBatch()
    dts = build_ensemble(b, api, specs, ntracers=8)
    b.configure(dts, "MUSCL", "PPM", "FCT")
    init = [[b.get_values(m, t) for t in range(1, 9)] for m in range(3)]
    yield b, specs, dts, init
    b.close()


def _state(b):
    return [[b.get_values(m, t) for t in range(1, 9)] for m in range(len(b.members))]


def _reset(b, init):
    for m, fields in enumerate(init):
        for t, v in enumerate(fields, start=1):
            b.set_values(m, t, v)


def _same(x, y):
    return all(np.array_equal(a, c) for fa, fc in zip(x, y) for a, c in zip(fa, fc))


def test_barrier_timeout_is_reported(lib):
    assert lib.tracer_selftest_barrier_timeout(1 << 14) == 1


@pytest.mark.parametrize("path", ["cooperative", "phases"])
def test_persistent_step_matches_separate_launches(small_batch, path):
    b, specs, dts, init = small_batch
    b.set_tile(cells_per_block=256, threads=128, blocks_per_sm=2, wave=1)
    b.set_path(path)
    assert b.path() == path
    b.steps(3, graph=True)
    graph = _state(b)
    _reset(b, init)
    b.steps(3, graph=False)
    plain = _state(b)
    _reset(b, init)
    b.steps_separate(3)
    sep = _state(b)
    _reset(b, init)
    b.steps_separate(3, graph=True)
    sep_graph = _state(b)
    assert _same(graph, plain)
    assert _same(graph, sep)
    assert _same(graph, sep_graph)
    assert not _same(graph, init)
    assert all(np.all(np.isfinite(v)) for f in graph for v in f)


def test_tiles_do_not_change_results(small_batch):
    b, specs, dts, init = small_batch
    results = []
    for path in ("cooperative", "phases"):
        for tile in ({"cells_per_block": 128, "threads": 64, "blocks_per_sm": 1, "wave": 1},
                     {"cells_per_block": 512, "threads": 256, "blocks_per_sm": 2, "wave": 2}):
            _reset(b, init)
            b.set_tile(**tile)
            b.set_path(path)
            b.steps(2, graph=True)
            results.append(_state(b))
    assert all(_same(results[0], r) for r in results[1:])


def test_paths_mixed_step_by_step(small_batch):
    """Odd step counts on one path, then the other (the task tables of both
    paths follow the buffer swaps), against separate launches."""
    b, specs, dts, init = small_batch
    b.set_tile(cells_per_block=256, threads=128, blocks_per_sm=2, wave=1)
    b.set_path("cooperative")
    b.steps(1, graph=True)
    b.set_path("phases")
    b.steps(3, graph=True)
    b.set_path("cooperative")
    b.steps(1, graph=False)
    b.set_path("phases")
    b.steps(2, graph=False)
    mixed = _state(b)
    _reset(b, init)
    b.steps_separate(7)
    assert _same(mixed, _state(b))


def test_new_velocity_is_picked_up(small_batch, api):
    """A member's velocity replaced between steps: the batch recomputes that
    member's edge volume fluxes (both paths, as the separate launches do)."""
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    b, specs, dts, init = small_batch
    s = specs[1]
    c = layered_flow_case(api, s["nx"], s["nl"], periodic=s["periodic"], seed=s["seed"])
    api.cleanup()
    out = {}
    for path in ("cooperative", "phases", "separate"):
        _reset(b, init)
        b.set_velocity(1, c.uv, c.w)
        if path == "separate":
            b.steps_separate(1)
            b.set_velocity(1, 0.5 * c.uv, 0.5 * c.w)
            b.steps_separate(2)
        else:
            b.set_path(path)
            b.steps(1, graph=True)
            b.set_velocity(1, 0.5 * c.uv, 0.5 * c.w)
            b.steps(2, graph=True)
        out[path] = _state(b)
    assert _same(out["cooperative"], out["separate"])
    assert _same(out["phases"], out["separate"])
    assert not _same(out["phases"], init)


def test_member_matches_single_mesh_fp32_engine(small_batch, api):
    """Member 0, tracer 1 against the single-mesh FP32 path (one tracer per
    launch there, four here: same arithmetic per cell)."""
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    b, specs, dts, init = small_batch
    b.steps(2, graph=True)
    got = b.get_values(0, 1)
    s = specs[0]
    api.cleanup()
    c = layered_flow_case(api, s["nx"], s["nl"], periodic=s["periodic"], seed=s["seed"])
    api.set_precision("fp32")
    api.allocate_tracers(1)
    api.set_values(1, init[0][0])
    api.set_scheme(1, "MUSCL", "PPM", "FCT")
    api.set_velocity(c.uv, c.w)
    api.set_ab_refresh(True)
    api.advect_steps(2, dts[0])
    ref = api.get_tracer_values(1)
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(got - ref)) <= 1e-6 * scale


def test_autotune_keeps_state_and_picks_a_tile(small_batch):
    b, specs, dts, init = small_batch
    before = _state(b)
    log = b.autotune(1)
    assert "best:" in log
    t = b.tile()
    assert t["cells_per_block"] in (256, 384, 512) and t["threads"] in (128, 256)
    assert b.path() in ("cooperative", "phases", "separate")
    assert _same(_state(b), before)
    b.steps(2, graph=True)
    # the per-member path releases its graph with the members' work arrays
    assert b.info()["graph"] == (b.path() != "separate")


def test_learned_flux_runs_on_the_member_path(small_batch, api):
    """The learned antidiffusive flux on every member: the batch switches to
    the per-member path (the persistent paths have no MLP phase and are
    refused), graph and direct launches agree bit for bit, the result differs
    from the plain scheme, and member 0's tracer 1 matches the single-mesh
    FP32 engine with the same parameters."""
    from fesom2_tracer_dwarf_b200.learned import trained_params
    from fesom2_tracer_dwarf_b200.workloads import layered_flow_case
    b, specs, dts, init = small_batch
    b.steps_separate(2)
    plain = _state(b)
    _reset(b, init)
    p = trained_params()
    b.learn_set(p, True)
    assert b.path() == "separate"
    with pytest.raises(RuntimeError):
        b.set_path("phases")
    with pytest.raises(RuntimeError):
        b.add_member(12, 12, 6, 4)
    b.steps(2, graph=False)
    learned = _state(b)
    _reset(b, init)
    b.steps(2, graph=True)
    assert _same(learned, _state(b))
    assert not _same(learned, plain)
    assert all(np.all(np.isfinite(v)) for f in learned for v in f)
    got = learned[0][0]
    s = specs[0]
    api.cleanup()
    c = layered_flow_case(api, s["nx"], s["nl"], periodic=s["periodic"], seed=s["seed"])
    api.set_precision("fp32")
    api.allocate_tracers(1)
    api.set_values(1, init[0][0])
    api.set_scheme(1, "MUSCL", "PPM", "FCT")
    api.set_velocity(c.uv, c.w)
    api.set_ab_refresh(True)
    assert api.lib.tracer_learn_set(p.ctypes.data, 1) == 0
    api.advect_steps(2, dts[0])
    ref = api.get_tracer_values(1)
    assert np.max(np.abs(got - ref)) <= 1e-6 * np.max(np.abs(ref))
    b.learn_set(None, False)
    b.set_path("phases")
    assert b.path() == "phases"
