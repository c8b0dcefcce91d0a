"""The per-step epilogues of the captured RK3 step (RK.cuh:164-180): the
physical time (sum of each step's last-stage dt) and step count, the monitor
points (Monitor.cu:196-251: chosen bv / sv planes and the time per step in a
ring of `capacity` steps) and the statistics sums (StatisticsCollector.cu:
14-52: bv, bv^2, bv^3, bv^4, uv, uw, vw, Y_k per cell for the steps after the
start step), against the states downloaded after every step."""
import numpy as np
import pytest

import ostc

pytestmark = pytest.mark.gpu


def _interior(a, g):
    return a[..., g:a.shape[-3] - g, g:a.shape[-2] - g, g:a.shape[-1] - g]


def test_physical_time_and_step_count():
    case = ostc.case_mixing_layer(24, 20, 8)
    s, blocks = case.solver()
    s.initialize()
    _, dt = s.rk3_steps(6, history=True)
    t, n = s.physical_time()
    acc = 0.0
    for v in dt:
        acc += float(v)
    assert n == 6 and t == acc
    s.initialize()
    assert s.physical_time() == (0.0, 0)
    s.close()


@pytest.mark.parametrize("capacity", [8, 3])
def test_monitor_records_match_states(capacity):
    case = ostc.case_mixing_layer(24, 20, 8)
    s, blocks = case.solver()
    s.initialize()
    pts = [(0, 3, 4, 2), (0, 23, 19, 7), (0, 10, 10, 0)]
    s.set_monitor(pts, bv_labels=(0, 1, 4, 5), sv_labels=(0, 8), capacity=capacity)
    g = blocks[0].ngg
    states, times = [], []
    for step in range(5):
        s.rk3_steps(1)
        bv, sv = blocks[0].download("bv"), blocks[0].download("sv")
        states.append([[bv[l, k + g, j + g, i + g] for l in (0, 1, 4, 5)] + [sv[l, k + g, j + g, i + g] for l in (0, 8)]
                       for (_, i, j, k) in pts])
        times.append(s.physical_time()[0])
    rec = s.get_monitor()
    assert rec.shape == (len(pts), min(5, capacity), 7)
    for step in range(5):
        if step < 5 - capacity:
            continue  # overwritten in the ring
        slot = step % capacity
        for p in range(len(pts)):
            assert np.array_equal(rec[p, slot, :6], np.array(states[step][p]))
            assert rec[p, slot, 6] == times[step]
    # the ring restarts after a read
    s.rk3_steps(2)
    assert s.get_monitor().shape == (len(pts), 2, 7)
    s.set_monitor([])
    s.close()


def test_monitor_across_blocks_batched():
    lay = ostc.block_layout(5, dims=(40, 30, 32), ranges=((8, 20), (8, 14), (8, 10)), anchors=False)
    case = ostc.case_uneven_blocks(layout=lay, rans_model=2)
    s, blocks = case.solver()
    assert s.batching()
    s.initialize()
    pts = [(b, 2, 3, 1) for b in range(0, len(blocks), 3)]
    s.set_monitor(pts, bv_labels=(5,), sv_labels=(0, 1), capacity=4)
    s.rk3_steps(2)
    rec = s.get_monitor()
    for q, (b, i, j, k) in enumerate(pts):
        g = blocks[b].ngg
        bv, sv = blocks[b].download("bv"), blocks[b].download("sv")
        assert rec[q, 1, 0] == bv[5, k + g, j + g, i + g]
        assert rec[q, 1, 1] == sv[0, k + g, j + g, i + g] and rec[q, 1, 2] == sv[1, k + g, j + g, i + g]
    s.close()


def test_statistics_sums_match_states():
    case = ostc.case_mixing_layer(24, 20, 8)
    s, blocks = case.solver()
    s.initialize()
    s.set_statistics(True, start_step=2)
    g = blocks[0].ngg
    ref = {"s12": 0.0, "s34": 0.0, "srs": 0.0, "syk": 0.0}
    for step in range(1, 6):
        s.rk3_steps(1)
        if step <= 2:
            continue
        bv = _interior(blocks[0].download("bv"), g)
        sv = _interior(blocks[0].download("sv"), g)
        ref["s12"] = ref["s12"] + np.concatenate([bv, bv * bv])
        ref["s34"] = ref["s34"] + np.concatenate([bv * bv * bv, bv * bv * bv * bv])
        ref["srs"] = ref["srs"] + np.stack([bv[1] * bv[2], bv[1] * bv[3], bv[2] * bv[3]])
        ref["syk"] = ref["syk"] + sv[:9]
    st = s.get_statistics(0)
    assert st["count"] == 3
    for got, key in ((st["sum12"], "s12"), (st["sum34"], "s34"), (st["sum_rs"], "srs"), (st["sum_yk"], "syk")):
        r = ref[key]
        for l in range(r.shape[0]):
            den = np.max(np.abs(r[l])) or 1.0
            assert np.max(np.abs(got[l] - r[l])) <= 1e-14 * den, (key, l)
    s.set_statistics(False)
    s.close()


def test_restart_from_checkpoint_continues_the_run():
    """a checkpoint (bv, sv of the caller's arrays plus physical time and step)
    restored into a fresh context continues the run: after 3 + 3 steps the
    state matches 6 uninterrupted steps to round-off (cv is rebuilt from bv at
    the restart, as the reference's read_flowfield does), the clock exactly.
    Faces that rebuild their ghost cv each stage only: symmetry and far-field
    ghosts keep the cv of the run's start (quirk A5), which a restart resets"""
    case = ostc.case_vortex(40, 32, 8, steps=6)
    for f in case.faces:
        if f.type_label == ostc.BC_SYMMETRY:
            f.type_label = ostc.BC_OUTFLOW
    s, blocks = case.solver()
    s.initialize()
    s.rk3_steps(6)
    ref_bv = blocks[0].download("bv")
    ref_t, ref_n = s.physical_time()
    s.close()
    s1, b1 = case.solver()
    s1.initialize()
    s1.rk3_steps(3)
    ckpt = {n: b1[0].download(n) for n in ("bv",)}
    t3, n3 = s1.physical_time()
    s1.close()
    host = case.blocks[0].copy()
    host.arrays["bv"][...] = ckpt["bv"]
    s2, b2 = ostc.Case(case.name, case.scheme, case.mech, [host], case.faces, 3).solver()
    s2.initialize()
    s2.set_physical_time(t3, n3)
    s2.rk3_steps(3)
    got = b2[0].download("bv")
    for l in range(6):
        den = np.max(np.abs(ref_bv[l])) or 1.0
        assert np.max(np.abs(got[l] - ref_bv[l])) <= 1e-12 * max(den, np.max(np.abs(ref_bv[1]))), l
    t, n = s2.physical_time()
    assert n == ref_n == 6 and abs(t - ref_t) <= 1e-15 * ref_t
    s2.close()
