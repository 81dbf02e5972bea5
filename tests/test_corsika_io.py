"""CORSIKA photon files: the package's EventIO and event-tape readers
against merlict's own (eventio::Run, event_tape::Run, compiled into the
harness), on merlict's test files and on files written here, and against
the known answers of merlict's EventIoTest.cpp."""
import os
import struct

import numpy as np
import pytest

from merlict_development_kit_b200 import corsika_io as CI
from oracle import oracle as O

needs_ref = pytest.mark.skipif(not O.harness_available(), reason="reference harness not built")
RESOURCES = os.path.join(O.REFERENCE_DIR, "merlict_corsika", "tests", "resources")
TELESCOPE_DAT = os.path.join(RESOURCES, "telescope.dat")
EVENT_TAPE = os.path.join(RESOURCES, "run_event_tape.tar")
needs_files = pytest.mark.skipif(not (os.path.exists(TELESCOPE_DAT) and os.path.exists(EVENT_TAPE)),
                                 reason="merlict's CORSIKA test files are not here")


# ---- an EventIO writer for fixtures (the layout eventio.cpp reads) -------------------

def _top(typ, ident, payload, version=0, only_sub=False):
    length = len(payload) | ((1 << 30) if only_sub else 0)
    return struct.pack("<iiii", CI.SYNC, typ | (version << 20), ident, length) + payload


def _sub(typ, ident, payload, version=0):
    return struct.pack("<iii", typ | (version << 20), ident, len(payload)) + payload


def _block273(values, n=273):
    return struct.pack("<i", n) + np.asarray(values, dtype="<f4").tobytes()


def write_eventio(path, events, compact_every=2, seed=0):
    """events: list of lists of bunch arrays [n][8] (one per telescope)."""
    rng = np.random.default_rng(seed)
    runh = CI.header_block("RUNH", {1: 42, 15: -2.0, 16: 10.0, 17: 100.0, 4: 1, 5: 5e5})
    out = _top(1200, 42, _block273(runh))
    out += _top(1212, 42, b"RUNNR 42\nEVTNR 1\n" + b" " * 64)
    tel = np.array([[0, 0, 500, 400], [1000, -200, 500, 400]], dtype="<f4")
    out += _top(1201, 42, struct.pack("<i", len(tel)) + tel.T.copy().tobytes())
    for e, tels in enumerate(events, start=1):
        evth = CI.header_block("EVTH", {1: e, 2: 1, 3: 1000.0 + e, 43: 42})
        out += _top(1202, e, _block273(evth))
        off = struct.pack("<if", len(tels), 123.5) + rng.normal(size=len(tels)).astype("<f4").tobytes() \
            + rng.normal(size=len(tels)).astype("<f4").tobytes()
        out += _top(1203, e, off)
        subs = b""
        for t, b in enumerate(tels):
            b = np.asarray(b, dtype=np.float32).reshape(-1, 8)
            if (t + e) % compact_every == 0:
                c = np.empty_like(b, dtype=np.int16)
                c[:, 0] = np.round(b[:, 0] / 0.1)
                c[:, 1] = np.round(b[:, 1] / 0.1)
                c[:, 2] = np.round(b[:, 2] * 30000.)
                c[:, 3] = np.round(b[:, 3] * 30000.)
                c[:, 4] = np.round(b[:, 4] / 0.1)
                c[:, 5] = np.round(np.log10(np.maximum(b[:, 5], 1.0)) * 1000.)
                c[:, 6] = np.round(b[:, 6] / 0.01)
                c[:, 7] = np.round(b[:, 7])
                body = struct.pack("<hhfi", 0, t, float(b[:, 6].sum()), len(b)) + c.astype("<i2").tobytes()
                subs += _sub(1205, t, body, version=1000)
            else:
                body = struct.pack("<hhfi", 0, t, float(b[:, 6].sum()), len(b)) + b.astype("<f4").tobytes()
                subs += _sub(1205, t, body)
        out += _top(1204, e, subs, only_sub=True)
        out += _top(1209, e, _block273(CI.header_block("EVTE", {1: e})))
    out += _top(1210, 42, _block273(np.zeros(273), n=3)[:4 + 12])
    with open(path, "wb") as f:
        f.write(out)


def bunches(rng, n):
    b = np.empty((n, 8), dtype=np.float32)
    b[:, 0] = rng.uniform(-3000, 3000, n)
    b[:, 1] = rng.uniform(-3000, 3000, n)
    b[:, 2] = rng.uniform(-0.05, 0.05, n)
    b[:, 3] = rng.uniform(-0.05, 0.05, n)
    b[:, 4] = rng.uniform(0, 300, n)
    b[:, 5] = rng.uniform(5e5, 2e6, n)
    b[:, 6] = rng.uniform(0, 16, n)
    b[:, 7] = rng.uniform(250, 700, n)
    return b


def mine_eventio(path):
    run = CI.EventIoRun(path)
    evs = list(run)
    return run, evs


def compare_eventio(path):
    run, evs = mine_eventio(path)
    ref = O.corsika_file_reference(path, "eventio")
    assert np.array_equal(run.header, ref["run_header"])
    assert run.input_card == ref["input_card"]
    assert np.array_equal(run.telescope_positions.ravel(), ref["telescope_positions"])
    assert len(evs) == len(ref["bunch_start"]) - 1
    for k, e in enumerate(evs):
        a, b = ref["bunch_start"][k], ref["bunch_start"][k + 1]
        assert np.array_equal(e.photons.ravel(), ref["bunches"][8 * a:8 * b])
        assert np.array_equal(e.header, ref["event_headers"][273 * k:273 * (k + 1)])
        oa, ob = ref["offset_start"][k], ref["offset_start"][k + 1]
        assert np.array_equal(e.telescope_offsets.ravel(), ref["telescope_offsets"][4 * oa:4 * ob])
    return run, evs


def compare_tape(path):
    run = CI.EventTapeRun(path)
    evs = list(run)
    ref = O.corsika_file_reference(path, "event_tape")
    assert np.array_equal(run.header, ref["run_header"])
    assert len(evs) == len(ref["bunch_start"]) - 1
    for k, e in enumerate(evs):
        a, b = ref["bunch_start"][k], ref["bunch_start"][k + 1]
        assert np.array_equal(e.photons.ravel(), ref["bunches"][8 * a:8 * b])
        assert np.array_equal(e.header, ref["event_headers"][273 * k:273 * (k + 1)])
    return run, evs


# ---- merlict's test files ------------------------------------------------------------------

@needs_ref
@needs_files
def test_telescope_dat_matches_merlicts_reader():
    compare_eventio(TELESCOPE_DAT)


@needs_files
def test_telescope_dat_known_answers():
    """EventIoTest.cpp: the run and event headers of telescope.dat."""
    run, evs = mine_eventio(TELESCOPE_DAT)
    assert run.header[0] == np.float32(CI.chars_to_float("RUNH"))
    assert run.telescope_positions.tolist() == [[0.0, 0.0, 500.0, 500.0]]
    assert run.input_card[100] == " "
    assert run.header[1] == pytest.approx(7.0, abs=1e-6)               # run number
    assert run.header[15] == pytest.approx(-2.7, abs=1e-6)             # spectral slope
    assert run.header[16] == pytest.approx(1000.0, abs=1e-6)
    assert run.header[17] == pytest.approx(50000.0, abs=1e-6)
    assert int(run.header[4]) == 1                                     # observation levels
    assert run.header[5] == pytest.approx(220000.0, abs=1e-6)
    e = evs[0]
    assert e.telescope_offsets.shape == (1, 4)
    assert e.telescope_offsets[0, 0] == pytest.approx(379489.3125, abs=1e-6)
    assert e.telescope_offsets[0, 1] == pytest.approx(0.0, abs=1e-6)
    assert e.telescope_offsets[0, 2] == pytest.approx(-6589.96044922, abs=1e-6)
    assert e.header[1] == 1.0 and e.header[2] == 1.0
    assert e.header[3] == pytest.approx(2745.3125, abs=1e-6)
    assert e.photons.shape == (42629, 8)


@needs_ref
@needs_files
def test_merlicts_event_tape_matches_merlicts_reader():
    compare_tape(EVENT_TAPE)


# ---- files written here ------------------------------------------------------------------

@needs_ref
def test_eventio_files_written_here(tmp_path):
    rng = np.random.default_rng(7)
    events = [[bunches(rng, 300), bunches(rng, 17)], [bunches(rng, 0), bunches(rng, 1000)],
              [bunches(rng, 5)]]
    p = str(tmp_path / "run.eventio")
    write_eventio(p, events)
    run, evs = compare_eventio(p)
    # one event per bunch block, as eventio::Run hands them out
    assert [len(e.photons) for e in evs] == [300, 17, 0, 1000, 5]
    assert run.telescope_positions.shape == (2, 4)
    # full blocks come back as written (event 1, telescope 0), compact ones
    # as merlict decodes them: to the compact form's resolution
    assert np.array_equal(evs[0].photons, events[0][0])
    assert np.allclose(evs[1].photons[:, :2], events[0][1][:, :2], atol=0.051)
    assert np.allclose(evs[1].photons[:, 5], events[0][1][:, 5], rtol=2e-3)


@needs_ref
@pytest.mark.parametrize("buffer_size", [1, 7, 2 ** 16])
def test_event_tapes_written_here(tmp_path, buffer_size):
    rng = np.random.default_rng(buffer_size)
    p = str(tmp_path / "run.tar")
    w = CI.EventTapeWriter(p, buffer_size=buffer_size)
    w.write_runh(CI.header_block("RUNH", {1: 3}))
    sizes = [40, 0, 13, 250]
    written = []
    for e, n in enumerate(sizes, start=1):
        w.write_evth(CI.header_block("EVTH", {1: e, 43: 3}))
        b = bunches(rng, n)
        w.write_bunches(b)
        written.append(b)
    w.close()
    run, evs = compare_tape(p)
    assert [len(e.photons) for e in evs] == sizes
    for e, b in zip(evs, written):
        assert np.array_equal(e.photons, b)


@needs_ref
def test_event_tape_with_a_wrong_event_number_ends_early_in_both(tmp_path):
    p = str(tmp_path / "bad.tar")
    w = CI.EventTapeWriter(p)
    w.write_runh(CI.header_block("RUNH", {1: 3}))
    w.write_evth(CI.header_block("EVTH", {1: 1, 43: 3}))
    w.write_bunches(bunches(np.random.default_rng(1), 5))
    w.write_evth(CI.header_block("EVTH", {1: 2, 43: 3}))
    w.write_bunches(bunches(np.random.default_rng(2), 5))
    w.close()
    # rename the second event's block so that its number no longer matches
    import tarfile
    q = str(tmp_path / "bad2.tar")
    with tarfile.open(p) as src, tarfile.open(q, "w:", format=tarfile.USTAR_FORMAT) as dst:
        for m in src:
            data = src.extractfile(m).read()
            if m.name.endswith("000000002/000000001.cer.x8.float32"):
                m.name = m.name.replace("/000000001.cer", "/000000002.cer")
            import io
            dst.addfile(m, io.BytesIO(data))
    run, evs = compare_tape(q)
    assert len(evs) == 1 and run.error is not None


def test_missing_files_raise(tmp_path):
    with pytest.raises(RuntimeError):
        CI.EventIoRun(str(tmp_path / "none.dat"))
    with pytest.raises(RuntimeError):
        CI.EventTapeRun(str(tmp_path / "none.tar"))
