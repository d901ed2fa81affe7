"""Reader of the binary dumps written by tests/cpp/scenarios.h (dump_results)."""
from __future__ import annotations

import numpy as np


class Dump:
    def __init__(self, path):
        b = open(path, "rb").read()
        assert b[:4] == b"GFD1", path
        self._b = b
        self._o = 4
        self.P = self._i()
        S = self._i()
        self.samples = []
        for _ in range(S):
            gen = self._i()
            M = self._i()
            Nc = self._ia(self.P)
            ext = self._ia(self.P)
            freq = self._fa(self.P * M).reshape(self.P, M)
            self.samples.append({"generation": gen, "M": M, "Nc": Nc, "extinct": ext, "freq": freq})
        A = self._i()
        self.ids = self._ia(4 * A).reshape(A, 4)
        K = self._i()
        self.spectra = {}
        for _ in range(K):
            s, p, kind, n, ln = (self._i() for _ in range(5))
            self.spectra[(s, p, "sfs" if kind == 0 else "hist", n)] = self._fa(ln)

    def _i(self):
        v = int(np.frombuffer(self._b, dtype="<i4", count=1, offset=self._o)[0])
        self._o += 4
        return v

    def _ia(self, n):
        v = np.frombuffer(self._b, dtype="<i4", count=n, offset=self._o).copy()
        self._o += 4 * n
        return v

    def _fa(self, n):
        v = np.frombuffer(self._b, dtype="<f4", count=n, offset=self._o).copy()
        self._o += 4 * n
        return v
