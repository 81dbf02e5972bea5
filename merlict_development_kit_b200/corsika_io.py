"""CORSIKA photon files: the readers merlict feeds its photon factory from.

* EventIO, as CORSIKA's IACT option writes it (merlict_corsika/
  eventio.cpp): a run header (type 1200, 273 floats), the input card
  (1212), the telescope positions (1201), then per event its header
  (1202) and telescope offsets (1203), a telescope array (1204) holding
  photon-bunch blocks (1205, full float32 or the compact int16 form), the
  event end (1209), and the run end (1210).  `EventIoRun` walks a file the
  way eventio::Run does (eventio.cpp:288-415): at every step it tries a
  bunch block, an array header, an event header, an event end and a run
  end in that order, and one "event" is handed out per bunch block.
* The event tape (merlict_corsika/mli_corsika_EventTape_standalone.c:
  1265-1468): a tar of 'RRRRRRRRR/RUNH.float32',
  'RRRRRRRRR/EEEEEEEEE/EVTH.float32' and the event's bunch blocks
  'RRRRRRRRR/EEEEEEEEE/BBBBBBBBB.cer.x8.float32' (blocks counted from 1),
  with the reader's checks of names, sizes, the 'RUNH'/'EVTH' markers and
  the run and event numbers.  `EventTapeRun` mirrors event_tape::Run
  (event_tape.cpp:10-47); `EventTapeWriter` writes such a tape.

Bunches come out as float32 arrays [n][8] (x, y [cm], cx, cy, time [ns],
production height [cm], photons in the bunch, wavelength [nm]), the input
of `engine.Scene.corsika_photons` / mlgpu_corsika_photons.
"""
from __future__ import annotations

import io
import math
import re
import struct
import tarfile
from dataclasses import dataclass

import numpy as np

SYNC = -736130505                     # eventio.cpp:64-67
HEADER_FLOATS = 273


def chars_to_float(word: str) -> float:
    """The float whose four bytes spell `word` (corsika::str2float)."""
    return float(np.frombuffer(word.encode("ascii"), dtype="<f4")[0])


class NoSyncFound(RuntimeError):
    """eventio::NoSyncFoundException."""


class WrongType(RuntimeError):
    """eventio::WrongTypeException."""


@dataclass
class EventIoHeader:
    """eventio::Header (eventio.cpp:9-79)."""
    type: int
    version: int
    user: bool
    extended: bool
    only_sub_objects: bool
    length: int
    id: int


class _Stream:
    def __init__(self, data: bytes):
        self.data = data
        self.pos = 0

    def read(self, n: int) -> bytes:
        b = self.data[self.pos:self.pos + n]
        self.pos += n
        return b

    def i32(self, count: int = 1):
        b = self.read(4 * count)
        if len(b) < 4 * count:
            raise EOFError
        v = struct.unpack(f"<{count}i", b)
        return v if count > 1 else v[0]


def _read_header(s: _Stream, top_level: bool = True) -> EventIoHeader:
    start = s.pos
    try:
        if top_level:
            sync, typ, ident, length = s.i32(4)
            if sync != SYNC:
                s.pos = start
                raise NoSyncFound(f"Header 'sync' field not correct: {sync & 0xffffffff:x}")
        else:
            typ, ident, length = s.i32(3)
        t = typ & 0xffff
        version = (typ & 0xfff00000) >> 20
        user = bool(typ & (1 << 16))
        extended = bool(typ & (1 << 17))
        only_sub = bool(length & (1 << 30))
        ln = length & 0x3fffffff
        if extended:
            ext = s.i32() & 0xfff
            ln &= (ext << 12)           # Header::extend_length, eventio.cpp:52-61
    except EOFError:
        s.pos = start
        raise NoSyncFound("end of file") from None
    return EventIoHeader(t, version, user, extended, only_sub, ln, ident)


def _expect(s: _Stream, expect_type: int) -> EventIoHeader:
    """Run::__get_header (eventio.cpp:345-362): a top-level header of the
    given type, or the stream back where it was."""
    start = s.pos
    h = _read_header(s)
    if h.type != expect_type:
        s.pos = start
        raise WrongType(f"Expected header type: {expect_type} but actual it is {h.type}")
    return h


def _block_273(s: _Stream, expected_n: int = 273) -> np.ndarray:
    n = s.i32()
    if n != expected_n:
        raise RuntimeError(f"Expected first int32 to be {expected_n} but actual it is {n}")
    b = s.read(4 * HEADER_FLOATS)
    b = b + b"\0" * (4 * HEADER_FLOATS - len(b))
    return np.frombuffer(b, dtype="<f4").copy()


def _photon_block(s: _Stream) -> np.ndarray:
    """make_photons_from_stream (eventio.cpp:240-284)."""
    start = s.pos
    try:
        h = _read_header(s, top_level=False)
    except NoSyncFound:
        s.pos = start
        raise WrongType("end of file") from None
    if h.type != 1205:
        s.pos = start
        raise WrongType("not a photon bunch block")
    _array, _tel, _photons, n = struct.unpack("<hhfi", s.read(12))
    compact = h.version // 1000 == 1
    if compact:
        raw = np.frombuffer(s.read(16 * n), dtype="<i2").reshape(n, 8).astype(np.float32)
        b = raw.copy()
        b[:, 0] = (raw[:, 0].astype(np.float64) * 0.1).astype(np.float32)
        b[:, 1] = (raw[:, 1].astype(np.float64) * 0.1).astype(np.float32)
        b[:, 2] = (raw[:, 2].astype(np.float64) / 30000.).astype(np.float32)
        b[:, 3] = (raw[:, 3].astype(np.float64) / 30000.).astype(np.float32)
        b[:, 4] = (raw[:, 4].astype(np.float64) * 0.1).astype(np.float32)
        b[:, 5] = np.array([math.pow(10, float(v) * 0.001) for v in raw[:, 5]],
                           dtype=np.float64).astype(np.float32)
        b[:, 6] = (raw[:, 6].astype(np.float64) * 0.01).astype(np.float32)
        return b
    return np.frombuffer(s.read(32 * n), dtype="<f4").reshape(n, 8).copy()


@dataclass
class EventIoEvent:
    header: np.ndarray                  # 273 float32 (EVTH)
    telescope_offsets: np.ndarray       # [n][4] toff, xoff, yoff, weight
    photons: np.ndarray                 # [n][8] float32 bunches


class EventIoRun:
    """eventio::Run: the run header (`header`, `input_card`,
    `telescope_positions` [n][4] x, y, z, r), then events one bunch block
    at a time: `while run.has_still_events_left(): run.next_event()`."""

    def __init__(self, path: str):
        try:
            with open(path, "rb") as f:
                self._s = _Stream(f.read())
        except OSError:
            raise RuntimeError(f"Can not open file: {path}") from None
        self.path = path
        self.run_end_found = False
        s = self._s
        _expect(s, 1200)
        self.header = _block_273(s)
        h = _expect(s, 1212)
        self.input_card = s.read(h.length).decode("latin-1")
        h = _expect(s, 1201)
        ntel = s.i32()
        if ntel <= 0 or ((h.length - 4) // ntel) // 4 != 4:
            raise RuntimeError("telescope positions: expected 4 arrays")
        self.telescope_positions = np.frombuffer(s.read(16 * ntel), dtype="<f4").reshape(
            ntel, 4).copy()
        self._event_header = np.zeros(HEADER_FLOATS, dtype=np.float32)
        self._offsets = np.zeros((0, 4), dtype=np.float32)
        self.event_end = np.zeros(HEADER_FLOATS, dtype=np.float32)
        self.end = np.zeros(HEADER_FLOATS, dtype=np.float32)
        self._photons = self._next()

    def has_still_events_left(self) -> bool:
        return not self.run_end_found

    def next_event(self) -> EventIoEvent:
        e = EventIoEvent(self._event_header.copy(), self._offsets.copy(), self._photons)
        self._photons = self._next()
        return e

    def __iter__(self):
        while self.has_still_events_left():
            yield self.next_event()

    def _telescope_offsets(self, h: EventIoHeader) -> np.ndarray:
        s = self._s
        narray = s.i32()
        toff = struct.unpack("<f", s.read(4))[0]
        xoff = np.frombuffer(s.read(4 * narray), dtype="<f4")
        yoff = np.frombuffer(s.read(4 * narray), dtype="<f4")
        weight = np.ones(narray, dtype=np.float32)
        k = ((h.length - 8) // narray) // 4 if narray > 0 else 0
        if k == 3:
            weight = np.frombuffer(s.read(4 * narray), dtype="<f4").copy()
        elif k != 2:
            raise RuntimeError(f"num_following_arrays is {k} but only 2 or 3 are allowed.")
        out = np.empty((narray, 4), dtype=np.float32)
        out[:, 0] = toff
        out[:, 1] = xoff
        out[:, 2] = yoff
        out[:, 3] = weight
        return out

    def _next(self) -> np.ndarray:
        s = self._s
        while not self.run_end_found:
            found = False
            try:
                return _photon_block(s)
            except WrongType:
                pass
            for step in (self._array, self._event_header_step, self._event_end, self._run_end):
                try:
                    step()
                    found = True
                except (WrongType, NoSyncFound):
                    pass
            if not found:
                raise RuntimeError("Not a single valid structure found in file.")
        return np.zeros((0, 8), dtype=np.float32)

    def _array(self):
        _expect(self._s, 1204)

    def _event_header_step(self):
        _expect(self._s, 1202)
        self._event_header = _block_273(self._s)
        h = _expect(self._s, 1203)
        self._offsets = self._telescope_offsets(h)

    def _event_end(self):
        _expect(self._s, 1209)
        self.event_end = _block_273(self._s)

    def _run_end(self):
        _expect(self._s, 1210)
        self.end = _block_273(self._s, expected_n=3)
        self.run_end_found = True


# ---- the event tape ------------------------------------------------------------------

_RUNH = re.compile(r"^(\d{9})/RUNH\.float32$")
_EVTH = re.compile(r"^(\d{9})/(\d{9})/EVTH\.float32$")
_BLOCK = re.compile(r"^(\d{9})/(\d{9})/(\d{9})\.cer\.x8\.float32$")


@dataclass
class EventTapeEvent:
    header: np.ndarray                  # 273 float32 (EVTH)
    photons: np.ndarray                 # [n][8] float32 bunches


class EventTapeRun:
    """event_tape::Run (event_tape.cpp:10-47) over the checks of
    mliEventTapeReader (mli_corsika_EventTape_standalone.c:1265-1468)."""

    def __init__(self, path: str):
        try:
            self._tar = tarfile.open(path, "r:")
        except (OSError, tarfile.TarError):
            raise RuntimeError("Can't open event-tape for reading.") from None
        self._members = iter(self._tar)
        self._cur = next(self._members, None)
        m = self._cur
        if m is None:
            raise RuntimeError("Can't read RUNH from event-tape.")
        g = _RUNH.match(m.name)
        if not g or m.size != 4 * HEADER_FLOATS:
            raise RuntimeError("Can't read RUNH from event-tape.")
        self.header = self._floats(m)
        if self.header[0] != np.float32(chars_to_float("RUNH")):
            raise RuntimeError("Expected RUNH[0] == 'RUNH'")
        self.run_number = int(g.group(1))
        if self.run_number != int(round(float(self.header[1]))):
            raise RuntimeError("Expected run_number in RUNH's path to match run_number in RUNH.")
        self._cur = next(self._members, None)
        self._next_evth = self._read_evth()

    def _floats(self, m) -> np.ndarray:
        data = self._tar.extractfile(m).read()
        return np.frombuffer(data, dtype="<f4").copy()

    # A malformed EVTH or bunch block ends the run, as in event_tape::Run,
    # which treats the reader's failure like the end of the tape; `error`
    # says why.
    error: str | None = None

    def _read_evth(self):
        m = self._cur
        if m is None:
            return None
        g = _EVTH.match(m.name)
        if not g:
            return None
        if m.size != 4 * HEADER_FLOATS:
            self.error = "Expected EVTH to have size 273*sizeof(float)"
            return None
        evth = self._floats(m)
        if evth[0] != np.float32(chars_to_float("EVTH")):
            self.error = "Expected EVTH[0] == 'EVTH'"
            return None
        if int(evth[1]) != int(g.group(2)) or int(evth[43]) != int(g.group(1)):
            self.error = "Expected the path's run and event numbers to match the EVTH's."
            return None
        self._event_number = int(g.group(2))
        self._cur = next(self._members, None)
        if self._block_state(1) != "ok":
            self.error = "Expected cherenkov-bunch-block after EVTH."
            return None
        return evth

    def _block_state(self, number: int) -> str:
        """'ok', 'none' (not a bunch block: the event ends) or 'bad'."""
        m = self._cur
        if m is None or not _BLOCK.match(m.name):
            return "none"
        g = _BLOCK.match(m.name)
        if (int(g.group(1)) != self.run_number or int(g.group(2)) != self._event_number or
                int(g.group(3)) != number):
            self.error = "Cherenkov-bunch-block's tar-header doesn't match."
            return "bad"
        if m.size % 32 != 0:
            self.error = "Expected cherenkov-bunch-block-size to be multiple of bunch-size."
            return "bad"
        return "ok"

    def has_still_events_left(self) -> bool:
        return self._next_evth is not None

    def next_event(self) -> EventTapeEvent:
        header = self._next_evth
        blocks, number = [], 1
        state = self._block_state(number)
        while state == "ok":
            blocks.append(self._floats(self._cur).reshape(-1, 8))
            self._cur = next(self._members, None)
            number += 1
            state = self._block_state(number)
        self._next_evth = self._read_evth() if state == "none" else None
        photons = np.concatenate(blocks) if blocks else np.zeros((0, 8), dtype=np.float32)
        return EventTapeEvent(header, photons)

    def __iter__(self):
        while self.has_still_events_left():
            yield self.next_event()

    def close(self):
        self._tar.close()


class EventTapeWriter:
    """Writes an event tape: `write_runh`, then per event `write_evth` and
    its bunches (`write_bunches`, in blocks of `buffer_size` bunches)."""

    def __init__(self, path: str, buffer_size: int = 2 ** 16):
        self._tar = tarfile.open(path, "w:", format=tarfile.USTAR_FORMAT)
        self.buffer_size = int(buffer_size)
        self.run_number = 0
        self.event_number = 0
        self._block = 0
        self._buf: list = []

    def _add(self, name: str, data: bytes):
        ti = tarfile.TarInfo(name)
        ti.size = len(data)
        self._tar.addfile(ti, io.BytesIO(data))

    def write_runh(self, runh):
        self._flush()
        runh = np.asarray(runh, dtype="<f4")
        self.run_number = int(round(float(runh[1])))
        self._add(f"{self.run_number:09d}/RUNH.float32", runh.tobytes())

    def write_evth(self, evth):
        self._flush()
        evth = np.asarray(evth, dtype="<f4")
        if int(round(float(evth[43]))) != self.run_number:
            raise ValueError("Expected run_number in EVTH to match run_number in last RUNH.")
        self.event_number = int(round(float(evth[1])))
        self._add(f"{self.run_number:09d}/{self.event_number:09d}/EVTH.float32", evth.tobytes())
        self._block = 0
        self._buf = []
        self._open_event = True

    def write_bunches(self, bunches):
        for row in np.asarray(bunches, dtype="<f4").reshape(-1, 8):
            self._buf.append(row)
            if len(self._buf) == self.buffer_size:
                self._flush_block()

    def _flush_block(self):
        self._block += 1
        self._add(f"{self.run_number:09d}/{self.event_number:09d}/{self._block:09d}.cer.x8.float32",
                  np.asarray(self._buf, dtype="<f4").reshape(-1, 8).tobytes())
        self._buf = []

    def _flush(self):
        if getattr(self, "_open_event", False):
            if self._buf or self._block == 0:
                self._flush_block()
            self._open_event = False

    def close(self):
        self._flush()
        self._tar.close()


def header_block(marker: str, numbers: dict) -> np.ndarray:
    """A 273-float header whose word 0 is `marker` ('RUNH', 'EVTH', ...)
    and whose words numbers[k] are set (e.g. {1: run number})."""
    h = np.zeros(HEADER_FLOATS, dtype=np.float32)
    h[0] = chars_to_float(marker)
    for k, v in numbers.items():
        h[k] = v
    return h


__all__ = ["EventIoRun", "EventIoEvent", "EventTapeRun", "EventTapeEvent", "EventTapeWriter",
           "header_block", "chars_to_float", "NoSyncFound", "WrongType"]
