"""CPU emulation of the FP32 multigrid cycle inside FP64 FGMRES: the oracle's
reference-shaped MultiGrid (Galerkin hierarchy and ADLJ line factors built
in FP64) with every level operator, transfer operator and line factor
rounded to FP32 and the cycle's vectors kept in FP32; the coarsest dense
solve in FP64.  Test infrastructure for the pressure operator's pin signs."""
import numpy as np

import lsg_oracle as lo

F = np.float32


class MultiGridFP32(lo.MultiGrid):
    def __init__(self, A, dims, **kw):
        super().__init__(A, dims, **kw)
        for lv in self.levels:
            lv.A32 = lv.A.astype(F)
            if getattr(lv, "R", None) is not None:
                lv.R32, lv.P32 = lv.R.astype(F), lv.P.astype(F)
            lv.tri32 = {k: tuple(np.asarray(a, dtype=F) for a in v) for k, v in lv.tri.items()}

    @staticmethod
    def _thomas(c, d, e, rhs, L):
        nl = rhs.shape[0]
        Cl = np.concatenate([c, np.zeros(1, c.dtype)]).reshape(nl, L)
        Dl = d.reshape(nl, L)
        El = np.concatenate([e, np.zeros(1, e.dtype)]).reshape(nl, L)
        y = np.empty_like(rhs)
        y[:, 0] = rhs[:, 0] * Dl[:, 0]
        for t in range(1, L):
            y[:, t] = (rhs[:, t] - Cl[:, t - 1] * y[:, t - 1]) * Dl[:, t]
        for t in range(L - 2, -1, -1):
            y[:, t] -= El[:, t] * y[:, t + 1]
        return y

    def apply(self, b):
        L = len(self.levels) - 1
        rs = [np.asarray(b, dtype=F).copy()]
        for k in range(L):
            rs.append(self.levels[k].R32 @ rs[k])
        cHH = lo.coarse_solve(self.lu, rs[L].astype(np.float64)).astype(F)
        for k in range(L - 1, -1, -1):
            lv = self.levels[k]
            tri64, lv.tri = lv.tri, lv.tri32
            try:
                ch = lv.P32 @ cHH
                c = ch.copy()
                r = rs[k]
                for _ in range(self.n_post):
                    for dname in "zyx":
                        r -= lv.A32 @ c
                        c = self._tdma(lv, dname, r)
                        c *= F(self.omega)
                        ch += c
            finally:
                lv.tri = tri64
            cHH = ch
        return cHH.astype(np.float64)
