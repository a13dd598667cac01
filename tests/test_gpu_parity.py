"""Parity of the CUDA step with the FP64 oracle, stage by stage and over
trajectories (the reference's verify-dynamics.mjs replay and trajectory
gates, scripts/exoplasim-webgpu/). All run through the C ABI."""
import numpy as np
import pytest

import oracle
from tests.helpers import carbon_counter, copy_engine_to_oracle, field_names, pkg, planets, rel_rms, v3_gate

STAGES = ["gridpointa", "spectrala", "physics_in", "fixer", "surface_flux", "radiation", "precipitation",
          "surface", "carbon", "physics_out", "spectrald", "pack"]
# Per-step host values (inputs of every stage, written by the host), not outputs.
HOST_FIELDS = {"radiation_step", "surface_step", "carbon_step", "snapshot_step"}
# Transform and dynamics stages: besides V3, their outputs stay within the
# reference's 1e-5 relative RMS transform bound (verify-kernels.mjs:273).
DYNAMICS_STAGES = {"gridpointa", "spectrala", "spectrald"}
TRANSFORM_TOL = 1e-5
NHOR = {21: 2048, 42: 8192, 63: 18432}


def build(truncation, levels, seed=11, slots=1, mode=0, **kw):
    p = planets.make_planet(seed, truncation=truncation, levels=levels, **kw)
    e = pkg.Engine(truncation, levels, slots, mode=mode)
    for s in range(slots):
        e.configure(s, p)
    return p, e


@pytest.mark.gpu
@pytest.mark.parametrize("truncation,levels", [(21, 10), (21, 5), (42, 10), (63, 10)])
def test_initial_state_matches_oracle(truncation, levels):
    p, e = build(truncation, levels)
    m = oracle.model_for(p)
    for name, ref in m["state"].items():
        got = e.read(0, name).astype(np.float64)
        ref = np.asarray(ref, dtype=np.float64).reshape(-1)
        ref32 = ref.astype(np.float32).astype(np.float64)
        assert np.array_equal(got, ref32) or rel_rms(got, ref) < 1e-6, name


def replay_v3(p, truncation, levels, warm_steps, mode=0):
    """Per-stage replay judged by the reference's V3 gate
    (scripts/exoplasim-webgpu/verify-dynamics.mjs:13-59,179-204): the
    engine's state is copied into an FP64 and a sequential-f32 oracle before
    each stage, all three run the stage, and every field the stage changes
    is judged: the GPU's relative RMS error against FP64 at most twice the
    f32 oracle's, its count of points off by more than 1e-5 of the field's
    RMS at most twice the f32 count plus one, with the one-column outlier
    rule. Returns {(field, stage): verdict}."""
    e = pkg.Engine(truncation, levels, 1, mode=mode)
    e.configure(0, p)
    m = oracle.model_for(p)
    o64, o32 = oracle.Oracle(m), oracle.Oracle(m, precision=32)
    e.step(warm_steps)
    names = field_names(o64)
    out = {}
    for stage in STAGES:
        info = e.slot_info(0)
        before = {n: e.read(0, n) for n in names if n not in HOST_FIELDS}
        for o in (o64, o32):
            for n in names:
                o.set(n, before[n].astype(np.float64) if n in before else e.read(0, n).astype(np.float64))
            o.set_phase(info["startup_left"])
            o.carbon_step = carbon_counter(m, info["step"] - m["start_step"])
            o.write_step_values(info["step"], publish=True)
        e.run_stage(stage)
        o64.run(stage)
        o32.run(stage)
        for n in before:
            ref, got = o64.get(n), e.read(0, n)
            if np.array_equal(got, before[n]) and np.array_equal(ref, before[n].astype(np.float64)):
                continue  # the stage leaves the field alone
            out[(n, stage)] = v3_gate(got, ref, o32.get(n), NHOR[truncation])
            out[(n, stage)]["rel_rms"] = rel_rms(got, ref)
            out[(n, stage)]["ok4"] = v3_gate(got, ref, o32.get(n), NHOR[truncation], factor=4)["ok"]
    return out


# Stages whose outputs pass through the Legendre transforms; on the
# split-precision path (mode 2, tensor cores) their fields are held to the
# north star's 1e-5 bound, since 3xTF32 with the tensor cores' FP32
# accumulation is about 3x a sequential-f32 sum's error (V3 asks 2x).
TRANSFORM_STAGES = {"gridpointa", "physics_in", "precipitation", "physics_out", "spectrald"}
# The column physics the precipitation stage runs after its split-precision
# transform keeps V3's form at twice its factor (4x sequential f32).


@pytest.mark.gpu
@pytest.mark.parametrize("truncation,levels,warm,mode", [
    (21, 10, 6, 0), (21, 5, 6, 0), (42, 10, 4, 0), (63, 10, 4, 0),
    (21, 10, 6, 1), (21, 5, 6, 1), (42, 10, 4, 1), (63, 10, 4, 1),
    (21, 10, 6, 2), (42, 10, 4, 2), (63, 10, 4, 2)])
def test_stage_replay_passes_v3(truncation, levels, warm, mode):
    """Every field of every stage, the snapshot pack and the FP64 global sums
    (fixsum, ice_sums) included, passes V3 against the FP64 oracle with the
    sequential-f32 oracle as comparator; transform and dynamics outputs are
    also within 1e-5 relative RMS. On the split-precision path the fields of
    the transform stages are held to 1e-5 instead of V3."""
    verdicts = replay_v3(planets.make_planet(11, truncation=truncation, levels=levels), truncation, levels, warm,
                         mode)
    assert ("snapshot", "pack") in verdicts and ("fixsum", "fixer") in verdicts and ("ice_sums", "surface") in verdicts
    rows = sorted(((v["gpu"] / max(v["f32"], 1e-30), k, v) for k, v in verdicts.items()), key=lambda r: -r[0])
    print("V3 worst GPU/f32 error ratios:", [(f"{r:.2f}", k[0], k[1], f"{v['gpu']:.2e}", f"{v['f32']:.2e}",
                                              v["gpu_off"], v["f32_off"]) for r, k, v in rows[:12]])
    split = mode == 2
    failed = [(k, v) for k, v in verdicts.items() if not v["ok"] and not (split and k[1] in TRANSFORM_STAGES)]
    assert not failed, failed[:5]
    loose = [(k, v["rel_rms"]) for k, v in verdicts.items()
             if (k[1] in DYNAMICS_STAGES or (split and k[1] in TRANSFORM_STAGES and k[0] not in PHYSICS_OUTPUTS))
             and v["rel_rms"] > TRANSFORM_TOL]
    assert not loose, loose[:5]
    if split:  # the column physics behind a split-precision transform: V3 at twice its factor
        relaxed = [k for k, v in verdicts.items() if k[1] in TRANSFORM_STAGES and k[0] in PHYSICS_OUTPUTS
                   and not v["ok4"]]
        assert not relaxed, relaxed[:5]


# Physics outputs that the transform stages pass through unchanged but that
# carry the column physics' threshold sensitivity (precipitation's column
# kernels, physics_in's dimensional frame is transforms only).
PHYSICS_OUTPUTS = {"dtdt", "dqdt", "dcc", "dql", "dprc", "dprl", "dprs", "dqvi", "icclev", "icctot", "dprcl",
                   "dprll", "dca_dtdt", "dca_dqdt", "dca_limited", "dconv", "localprecip"}


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_global_sums_match_oracle(mode):
    """The fixer's and getiflx's per-planet FP64 sums (fixsum, ice_sums) are
    the oracle's sums of the same inputs, rounded once to f32: after each
    stage the engine's sums equal an FP64 sum of the engine's own inputs to
    1e-6, and the FP64 oracle's (its inputs recomputed) to 1e-5."""
    p, e = build(21, 10, seed=12, mode=mode)
    e.step(6)
    m = oracle.model_for(p)
    o = oracle.Oracle(m)
    names = field_names(o)
    for stage in ("physics_in", "fixer", "surface_flux", "radiation", "precipitation", "surface"):
        info = e.slot_info(0)
        copy_engine_to_oracle(e, 0, o, names)
        o.set_phase(info["startup_left"])
        o.carbon_step = 0
        o.write_step_values(info["step"], publish=True)
        e.run_stage(stage)
        o.run(stage)
    for sums, parts in (("fixsum", ("fixneg", "fixpos")), ("ice_sums", ("ice_part1", "ice_part2"))):
        got = e.read(0, sums).astype(np.float64)
        own = np.array([e.read(0, f).astype(np.float64).sum() for f in parts])
        ref = o.get(sums)
        assert np.all(np.abs(got - own) <= 1e-6 * np.maximum(np.abs(own), 1e-30)), (sums, got, own)
        assert np.all(np.abs(got - ref) <= 1e-5 * np.maximum(np.abs(ref), 1e-30)), (sums, got, ref)


# The fields of the reference's free-running gate (trajectory.mjs:9-15).
V4_FIELDS = ("sd", "sz", "st", "sq", "sp", "sdm", "szm", "stm", "sqm", "spm", "dt", "dq", "du", "dv", "dp", "dprc",
             "dprl", "dprs", "dcc", "dalb", "dswfl", "dlwfl", "dshfl", "dlhfl", "devap", "land_dts", "dsoilt",
             "dsnowz", "dwatc", "driver", "dcveg", "dcsoil", "dglac", "xts", "xiced", "xicec", "xsnow", "ysst",
             "sea_dts", "localavgprecip", "localavgweather", "localavgtemps")


def v4_judge(engine, o64, o32, fields=V4_FIELDS):
    """V4 (trajectory.mjs:67-79): each field's RMS difference from the FP64
    run at most twice the sequential-f32 run's; a field FP64 leaves at zero
    stays zero. Returns {field: (gpu, f32, ok)}."""
    out = {}
    for n in fields:
        if o64.size(n) < 0:
            continue
        ref = o64.get(n)
        scale = np.sqrt(np.mean(ref * ref))
        got = engine.read(0, n).astype(np.float64)
        if scale == 0:
            out[n] = (float(np.abs(got).max()), 0.0, bool(np.all(got == 0)))
            continue
        g = rel_rms(got, ref)
        f = rel_rms(o32.get(n), ref)
        out[n] = (g, f, g <= 2 * f)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_startup_day_passes_v4(mode):
    """The first day from the set-up state (3 start-up steps, then 32 steps;
    the reference's verify-startup.mjs), judged by V4 against both oracles."""
    p, e = build(21, 10, seed=21, mode=mode)
    m = oracle.model_for(p)
    m["state"] = {k: np.asarray(v, dtype=np.float64).astype(np.float32).astype(np.float64)
                  for k, v in m["state"].items()}
    for name, v in m["state"].items():
        e.write(0, name, v.astype(np.float32))
    o64, o32 = oracle.Oracle(m), oracle.Oracle(m, precision=32)
    e.step(3)
    e.step(32)
    for o in (o64, o32):
        o.advance(32)
    verdict = v4_judge(e, o64, o32)
    print("1-day GPU/f32 error ratios:", {k: f"{g / max(f, 1e-30):.2f}" for k, (g, f, _) in verdict.items()})
    bad = {k: v for k, v in verdict.items() if not v[2]}
    assert not bad, bad


@pytest.mark.gpu
@pytest.mark.parametrize("truncation,mode", [(21, 1), (42, 1), (63, 1), (21, 2), (42, 2), (63, 2)])
def test_fft_matches_dense_dft(truncation, mode):
    """The optimized paths' transforms (FFTs, latitude-pair Legendre; mode 2
    with sp2fc and sp2fcdmu on the tensor cores) give the plain path's: one
    gridpointa from the same state in both modes."""
    p = planets.make_planet(71, truncation=truncation, levels=10)
    plain = pkg.Engine(truncation, 10, 1, mode=0)
    fast = pkg.Engine(truncation, 10, 1, mode=mode)
    plain.configure(0, p)
    fast.configure(0, p)
    plain.step(4)
    for name in field_names(oracle.Oracle(oracle.model_for(p))):
        fast.write(0, name, plain.read(0, name))
    plain.run_stage("gridpointa")
    fast.run_stage("gridpointa")
    for name in ("gu", "gv", "gt", "gd", "gz", "gq", "gp", "gpj", "gpmt", "fgtn", "fgke", "fgvz", "sdt", "stt", "sqt"):
        err = rel_rms(fast.read(0, name), plain.read(0, name))
        assert err < 1e-5, f"{name}: {err:.2e}"


@pytest.mark.gpu
def test_batched_slots_match_alone_bitwise():
    a = planets.make_planet(31, truncation=21, levels=10)
    b = planets.make_planet(32, truncation=21, levels=10, rotationPeriodDays=3.0, pressureBar=2.0, co2Ppm=5000.0)
    batch = pkg.Engine(21, 10, 3)
    batch.configure(0, a)
    batch.configure(1, b)
    batch.configure(2, a)
    alone = pkg.Engine(21, 10, 1)
    alone.configure(0, a)
    for _ in range(3):
        batch.step(5)
        alone.step(5)
    for name in ("st", "sz", "sd", "sq", "sp", "dt", "dq", "dcc", "dprc"):
        x0, x2, y = batch.read(0, name), batch.read(2, name), alone.read(0, name)
        assert np.array_equal(x0, x2), name
        assert np.array_equal(x0, y), name
        assert not np.array_equal(x0, batch.read(1, name)), name


@pytest.mark.gpu
def test_checkpoint_round_trip_is_bit_exact():
    p, e = build(21, 5, seed=41)
    e.step(3)
    e.step(4)
    saved = e.checkpoint_save(0)
    assert saved.startswith(b"GCM-WEBGPU-STATE\n")
    e.step(5)
    ref = {n: e.read(0, n) for n in ("st", "sz", "sd", "sq", "sp", "dt", "xsst")}
    f = pkg.Engine(21, 5, 1)
    f.configure(0, p)
    f.checkpoint_load(0, saved)
    assert f.slot_info(0)["step"] == e.slot_info(0)["step"] - 5
    f.step(5)
    for n, v in ref.items():
        assert np.array_equal(f.read(0, n), v), n


@pytest.mark.gpu
def test_checkpoint_rejects_other_layout():
    p, e = build(21, 5, seed=42)
    e.step(3)
    saved = e.checkpoint_save(0)
    q, g = build(21, 10, seed=42)
    with pytest.raises(pkg.ExogcmError) as err:
        g.checkpoint_load(0, saved)
    assert err.value.code == -4
    with pytest.raises(pkg.ExogcmError):
        g.checkpoint_load(0, b"not a checkpoint")


@pytest.mark.gpu
def test_unstable_slot_is_flagged_and_others_unaffected():
    a = planets.make_planet(51, truncation=21, levels=5)
    e = pkg.Engine(21, 5, 2)
    e.configure(0, a)
    e.configure(1, a)
    ref = pkg.Engine(21, 5, 1)
    ref.configure(0, a)
    e.step(3)
    ref.step(3)
    st = e.read(1, "st")
    st[7] = np.nan
    e.write(1, "st", st)
    e.step(2)
    ref.step(2)
    flags = e.unstable()
    assert flags.tolist() == [False, True]
    assert np.array_equal(e.read(0, "st"), ref.read(0, "st"))


@pytest.mark.gpu
def test_snapshot_publishes_on_schedule():
    p, e = build(21, 10, seed=61)
    e.step(3, publish_every=4)  # start-up steps never publish
    assert e.snapshot(0)[0] == -1
    e.step(4, publish_every=4)
    step, snap = e.snapshot(0)
    assert step == 0
    assert snap.shape == (101, 2048)
    assert np.all(np.isfinite(snap))
    e.step(4, publish_every=4)
    step, snap = e.snapshot(0)
    assert step == 4
    dt = e.read(0, "dt").reshape(11, -1)
    # field 0 is the surface temperature at the publishing step; the state has moved 3 steps on
    assert np.all(np.abs(snap[0] - dt[10]) < 30)


@pytest.mark.gpu
def test_bulk_snapshot_copy_overlaps_the_next_step():
    """exogcm_snapshots_begin copies every slot's snapshot field while the
    caller steps on: the copy keeps the day it was started on, equal to the
    per-slot reads of that day, although the next step overwrites the field."""
    torch = pytest.importorskip("torch")
    e = pkg.Engine(21, 10, 3, mode=1)
    for s in range(3):
        e.configure(s, planets.make_planet(70 + s, truncation=21, levels=10))
    e.step(3, publish_every=4)
    e.step(4, publish_every=4)
    per_slot = e.field_size("snapshot")
    bulk = torch.empty(3 * per_slot, dtype=torch.float32, pin_memory=True).numpy()
    for day in range(2):
        ref = [e.snapshot(s)[1] for s in range(3)]
        e.snapshots_begin(bulk)
        e.step(4, publish_every=4)  # packs new snapshots over the field being copied
        e.snapshots_wait()
        got = bulk.reshape(101, 3, 2048)
        for s in range(3):
            assert np.array_equal(got[:, s, :], ref[s]), (day, s)
        assert not np.array_equal(e.snapshot(0)[1], ref[0])
    with pytest.raises(pkg.ExogcmError):
        e.snapshots_begin(bulk[:-1])


@pytest.mark.gpu
def test_autotuned_shapes_leave_results_unchanged():
    """The first engine of each shape (device, resolution, slots, mode) times
    its transform shapes at its first configure, later ones reuse them;
    engines of 1 and 3 slots may pick different ones, and the shared planet
    must still step identically."""
    p = planets.make_planet(81, truncation=21, levels=10)
    one = pkg.Engine(21, 10, 1, mode=1)
    three = pkg.Engine(21, 10, 3, mode=1)
    one.configure(0, p)
    for s in range(3):
        three.configure(s, p)
    for e in (one, three):
        t = e.tuning()
        assert t["fft_rows"] in (8, 16, 32)
        for group, tile in (t["sp2fc"], t["dv2uv"]):
            assert group in (1, 2, 4) and tile in (8, 16, 32)
        assert set(t["forward_tiles"].values()) <= {8, 16}
    print("tunings:", one.tuning(), three.tuning())
    one.step(3)
    three.step(3)
    one.step(8)
    three.step(8)
    for name in ("st", "sz", "sd", "sq", "sp", "fgt", "gu"):
        assert np.array_equal(one.read(0, name), three.read(2, name)), name


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_full_step_equals_its_stages_bitwise(mode):
    """exogcm_step runs the stages as one graph and skips work whose result no
    later kernel of the step reads: physics_in's zeroed tendencies (the fixer,
    surflx, vdiff and physics_out take the zeros unread) and, on the optimized
    path, the Fourier fields between fused transforms. After one step every
    other field equals the same stages run one at a time through
    exogcm_run_stage, which does that work, bit for bit."""
    from tests.helpers import oracle_field_list
    p = planets.make_planet(91, truncation=21, levels=10)
    whole, staged = pkg.Engine(21, 10, 1, mode=mode), pkg.Engine(21, 10, 1, mode=mode)
    for e in (whole, staged):
        e.configure(0, p)
        e.step(3)
        e.step(4)
    whole.step(1, publish_every=1)  # stage replay publishes, so the pack stage writes the snapshot
    for stage in STAGES:
        staged.run_stage(stage)
    scratch = {"fgt", "fgd", "fgz", "fgq", "fgp", "fgpj", "fdqt", "fzdekin"} if mode else set()
    names = [n for n in oracle_field_list() if n not in scratch]
    differ = [n for n in names if not np.array_equal(whole.read(0, n), staged.read(0, n))]
    assert not differ, differ
