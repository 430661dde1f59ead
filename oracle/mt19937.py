"""MT19937 restatement used by the oracle to make seeded resampling uniforms.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product path.

Follows the reference's Fortran 95 port of Matsumoto & Nishimura's MT19937
(letkf/run/src/common_mt19937ar.f90): ``init_genrand`` (:130-156),
``genrand_int32`` (:211-265) and ``genrand_res53`` (:337-359), plus the
wrapper ``com_rand_seed`` (letkf/run/src/common.f90:1066-1095).  Vectorised
over independent seeds: state arrays have shape [nseeds, 624].

Pinned against the published MT19937 known answer (the 10000th output of
``init_genrand(5489)`` is 4123659995, the value the C++ standard requires of
std::mt19937) and against numpy's legacy ``RandomState`` (the same algorithm,
independent code) in tests/test_oracle_mt19937.py.
"""
from __future__ import annotations

import numpy as np

N, M = 624, 397
MATRIX_A = np.uint32(0x9908B0DF)
UPPER, LOWER = np.uint32(0x80000000), np.uint32(0x7FFFFFFF)


def init_genrand(seeds) -> np.ndarray:
    """State [nseeds, 624] for each 32-bit seed (common_mt19937ar.f90:130-156)."""
    s = np.atleast_1d(np.asarray(seeds, dtype=np.int64)).astype(np.uint64) & np.uint64(0xFFFFFFFF)
    mt = np.empty((s.size, N), dtype=np.uint32)
    mt[:, 0] = s.astype(np.uint32)
    prev = s
    for i in range(1, N):
        # mt(i) = 1812433253 * (mt(i-1) ^ (mt(i-1) >> 30)) + (i-1)   [1-based i]
        prev = (np.uint64(1812433253) * (prev ^ (prev >> np.uint64(30))) + np.uint64(i)) & np.uint64(0xFFFFFFFF)
        mt[:, i] = prev.astype(np.uint32)
    return mt


def _twist(mt: np.ndarray) -> None:
    """Regenerate all 624 words in place (common_mt19937ar.f90:228-256)."""
    for kk in range(N):
        y = (mt[:, kk] & UPPER) | (mt[:, (kk + 1) % N] & LOWER)
        mag = np.where((y & np.uint32(1)) != 0, MATRIX_A, np.uint32(0))
        mt[:, kk] = mt[:, (kk + M) % N] ^ (y >> np.uint32(1)) ^ mag


class MT19937Batch:
    """Independent MT19937 streams, one per seed."""

    def __init__(self, seeds):
        self.mt = init_genrand(seeds)
        self.mti = N

    def int32(self) -> np.ndarray:
        """Next tempered output of every stream (common_mt19937ar.f90:211-265)."""
        if self.mti >= N:
            _twist(self.mt)
            self.mti = 0
        y = self.mt[:, self.mti].copy()
        self.mti += 1
        y ^= y >> np.uint32(11)
        y ^= (y << np.uint32(7)) & np.uint32(0x9D2C5680)
        y ^= (y << np.uint32(15)) & np.uint32(0xEFC60000)
        y ^= y >> np.uint32(18)
        return y

    def res53(self) -> np.ndarray:
        """Uniform [0,1) with 53-bit resolution (common_mt19937ar.f90:337-359).

        The Fortran sums a1/2^11 + a0/2^27 + b1/2^37 + b0/2^53 of the 16-bit
        halves of a = int32 >> 5 and b = int32 >> 6; every partial sum is
        exact in binary64, so the value equals (a*2^26 + b) / 2^53.
        """
        a = (self.int32() >> np.uint32(5)).astype(np.float64)
        b = (self.int32() >> np.uint32(6)).astype(np.float64)
        return (a * 67108864.0 + b) / 9007199254740992.0


def com_rand_seed(ndim: int, seeds) -> np.ndarray:
    """rand(ndim) for each seed: init_genrand(seed), then ndim genrand_res53
    draws (letkf/run/src/common.f90:1066-1095 with iseed /= 0).  [nseeds, ndim]."""
    g = MT19937Batch(seeds)
    out = np.empty((g.mt.shape[0], ndim), dtype=np.float64)
    for i in range(ndim):
        out[:, i] = g.res53()
    return out


def pf_seed(point: np.ndarray, draw: np.ndarray, base: int = 0) -> np.ndarray:
    """Seed of the MT stream of (grid point, resampling draw).

    The reference seeds every draw from the wall clock (common.f90:1082-1084);
    reproducible runs replace that with this fixed map, shared by the oracle
    and the tests: seed = base + point * 131 + draw + 1 (mod 2^31)."""
    return (np.int64(base) + point.astype(np.int64) * 131 + draw.astype(np.int64) + 1) % (2 ** 31)
