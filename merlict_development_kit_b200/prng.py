"""merlict::random::Mt19937 on the host (merlict/random/Mt19937.cpp:8-33).

merlict draws from the C++ standard library's std::mt19937_64 and maps
each 64-bit word w to uniform() = double(w) * (1 / double(2^64 - 1)).
This module restates the published 64-bit Mersenne Twister (Matsumoto and
Nishimura, "Mersenne Twister 64-bit", 2004; the parameters the C++
standard fixes for std::mt19937_64) with numpy: the twist of the 312-word
state runs as three vector passes, the tempering over whole blocks, so a
million draws take milliseconds.  The words are bit-identical to the
standard library's, and so are the uniforms (numpy's uint64 -> float64
conversion rounds to nearest like the C++ static_cast).

The photon sources of merlict's JSON reader seed it with 0
(merlict_json/json.cpp:521-541), which is why it lives here: it decides
which photons a JSON "point_source" or "parallel_disc" makes.
"""
from __future__ import annotations

import numpy as np

_N, _M = 312, 156
_A = np.uint64(0xB5026F5AA96619E9)
_UPPER = np.uint64(0xFFFFFFFF80000000)
_LOWER = np.uint64(0x000000007FFFFFFF)
_F = 6364136223846793005
_MASK64 = (1 << 64) - 1
# 1.0/double(2^64 - 1): the divisor rounds to 2^64, so this is 2^-64
INV_MAX = 1.0 / float(_MASK64)


class Mt19937:
    """std::mt19937_64 with merlict's uniform() mapping."""

    def __init__(self, seed: int = 0):
        self.set_seed(seed)

    def set_seed(self, seed: int):
        mt = [0] * _N
        mt[0] = int(seed) & _MASK64
        for i in range(1, _N):
            prev = mt[i - 1]
            mt[i] = (_F * (prev ^ (prev >> 62)) + i) & _MASK64
        self._state = np.array(mt, dtype=np.uint64)
        self._index = _N
        self.seed = int(seed)

    def getstate(self):
        return (self._state.copy(), self._index, self.seed)

    def setstate(self, state):
        self._state, self._index, self.seed = state[0].copy(), int(state[1]), int(state[2])

    def _twist(self):
        mt = self._state
        one = np.uint64(1)

        def step(lo, hi, nxt, far):
            y = (mt[lo:hi] & _UPPER) | (nxt & _LOWER)
            mag = np.where((y & one) != 0, _A, np.uint64(0))
            mt[lo:hi] = far ^ (y >> one) ^ mag

        # i in [0, N-M): every operand is still the old state
        step(0, _N - _M, mt[1:_N - _M + 1].copy(), mt[_M:_N].copy())
        # i in [N-M, N-1): mt[i+M-N] was updated by the first pass
        step(_N - _M, _N - 1, mt[_N - _M + 1:_N].copy(), mt[0:_M - 1].copy())
        # i = N-1 wraps around to the already updated mt[0]
        step(_N - 1, _N, mt[0:1].copy(), mt[_M - 1:_M].copy())
        self._index = 0

    @staticmethod
    def _temper(y: np.ndarray) -> np.ndarray:
        y = y ^ ((y >> np.uint64(29)) & np.uint64(0x5555555555555555))
        y = y ^ ((y << np.uint64(17)) & np.uint64(0x71D67FFFEDA60000))
        y = y ^ ((y << np.uint64(37)) & np.uint64(0xFFF7EEE000000000))
        return y ^ (y >> np.uint64(43))

    def words(self, n: int) -> np.ndarray:
        """The next n 64-bit outputs of the engine."""
        out = np.empty(int(n), dtype=np.uint64)
        k = 0
        while k < n:
            if self._index >= _N:
                self._twist()
            take = min(n - k, _N - self._index)
            out[k:k + take] = self._temper(self._state[self._index:self._index + take])
            self._index += take
            k += take
        return out

    def uniforms(self, n: int) -> np.ndarray:
        """The next n values of merlict's uniform() (Mt19937.cpp:18-20)."""
        return self.words(n).astype(np.float64) * INV_MAX

    def uniform(self) -> float:
        return float(self.uniforms(1)[0])
