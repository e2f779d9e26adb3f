"""CPU oracle for the BEAGLE likelihood hot path: a float64 numpy restatement.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg may import this module, and only as the checker
(or the timed CPU baseline).  The product path never calls it.

The class below restates, vectorised over site patterns, what the reference
CPU implementation (``BeagleCPUImpl<double,1,0>``) computes for each API call
on the path.  Each method cites the reference file:line it follows (paths are
relative to the beagle-lib source tree).  Parity of this restatement is pinned
against the compiled reference library (``oracle/_ref``, built by
``oracle/Makefile``) by ``tests/test_oracle.py`` and by the golden fixtures in
``tests/golden/`` that ``tests/golden/make_golden.py`` produced by running the
compiled reference.

Layouts follow the reference CPU layout: partials ``[category][pattern][state]``,
transition matrices ``[category][state_i][state_j + pad]`` with one pad column
(T_PAD = 1, ``CPU/BeagleCPUImpl.h:43``), scale buffers ``[pattern]``.
"""

import numpy as np

# Flag bits and op constants with the values of libhmsbeagle/beagle.h:110-205.
SUCCESS = 0
ERROR_GENERAL = -1
ERROR_OUT_OF_RANGE = -5
ERROR_NO_IMPLEMENTATION = -7
ERROR_FLOATING_POINT = -8
OP_NONE = -1
FLAG_PRECISION_SINGLE = 1 << 0
FLAG_PRECISION_DOUBLE = 1 << 1
FLAG_SCALERS_RAW = 1 << 9
FLAG_SCALERS_LOG = 1 << 10
FLAG_INVEVEC_STANDARD = 1 << 20
FLAG_INVEVEC_TRANSPOSED = 1 << 21


class OracleInstance:
    """One BEAGLE instance, restated in float64 numpy.

    Mirrors ``BeagleCPUImpl::createInstance`` (``CPU/BeagleCPUImpl.hpp:234-490``)
    for the manual-scaling, real-eigen configuration used on the hot path.
    """

    def __init__(self, tipCount, partialsBufferCount, compactBufferCount,
                 stateCount, patternCount, eigenBufferCount, matrixBufferCount,
                 categoryCount, scaleBufferCount, flags=0):
        self.N = tipCount
        self.nbuf = partialsBufferCount + compactBufferCount
        self.S = stateCount
        self.P = patternCount
        self.C = categoryCount
        self.nmat = matrixBufferCount
        self.neig = eigenBufferCount
        # CPU/BeagleCPUImpl.hpp:307-313: SCALERS_LOG if asked for, else RAW.
        self.log_scalers = bool(flags & FLAG_SCALERS_LOG)
        self.invevec_transposed = bool(flags & FLAG_INVEVEC_TRANSPOSED)
        self.partials = [None] * self.nbuf
        self.states = [None] * self.nbuf
        for b in range(tipCount, self.nbuf):
            self.partials[b] = np.zeros((self.C, self.P, self.S))
        self.matrices = [np.zeros((self.C, self.S, self.S + 1)) for _ in range(self.nmat)]
        self.scale = [np.zeros(self.P) for _ in range(scaleBufferCount)]
        self.cube = [None] * eigenBufferCount
        self.evals = [None] * eigenBufferCount
        self.freqs = [None] * eigenBufferCount
        self.catw = [None] * eigenBufferCount
        self.rates = [None] * eigenBufferCount
        self.patw = np.ones(self.P)
        self.site_lnl = np.zeros(self.P)
        self.site_d1 = np.zeros(self.P)

    # ---- data in ---------------------------------------------------------
    def setTipStates(self, tip, states):
        """CPU/BeagleCPUImpl.hpp:570-584: states >= S become the missing state S."""
        s = np.asarray(states, dtype=np.int64).copy()
        s[s >= self.S] = self.S
        self.states[tip] = s

    def setTipPartials(self, tip, partials):
        """CPU/BeagleCPUImpl.hpp:587-618: one [P][S] block, copied to every category."""
        p = np.asarray(partials, dtype=np.float64).reshape(self.P, self.S)
        self.partials[tip] = np.broadcast_to(p, (self.C, self.P, self.S)).copy()

    def setPartials(self, buf, partials):
        """CPU/BeagleCPUImpl.hpp:678-706: full [C][P][S] block."""
        self.partials[buf] = np.asarray(partials, dtype=np.float64).reshape(
            self.C, self.P, self.S).copy()

    def setRootPrePartials(self, bufs, freq_idx, check=True):
        """CPU/BeagleCPUImpl.hpp:621-676: buffer = state frequencies in every
        category and pattern."""
        for b, f in zip(bufs, freq_idx):
            self.partials[b] = np.broadcast_to(self.freqs[f], (self.C, self.P, self.S)).copy()
        return SUCCESS

    def getPartials(self, buf, scaleIndex=OP_NONE):
        """CPU/BeagleCPUImpl.hpp:709-748.  With a cumulative scale index the
        reference multiplies only the first P*S entries (category 0) by
        exp(cumulative[p]); that behaviour is reproduced as is."""
        out = self.partials[buf].copy()
        if scaleIndex != OP_NONE:
            out[0] *= np.exp(self.scale[scaleIndex])[:, None]
        return out.reshape(-1)

    def setEigenDecomposition(self, e, evec, ivec, evals):
        """CPU/EigenDecompositionCube.hpp:69-100: cube C[i][j][k] = V[i][k] * Vinv[k][j]
        (Vinv read transposed under INVEVEC_TRANSPOSED)."""
        S = self.S
        V = np.asarray(evec, dtype=np.float64).reshape(S, S)
        Vi = np.asarray(ivec, dtype=np.float64).reshape(S, S)
        if self.invevec_transposed:
            Vi = Vi.T
        self.cube[e] = V[:, None, :] * Vi.T[None, :, :]          # [i][j][k]
        self.evals[e] = np.asarray(evals, dtype=np.float64).copy()

    def setStateFrequencies(self, i, f):
        self.freqs[i] = np.asarray(f, dtype=np.float64).copy()

    def setCategoryWeights(self, i, w):
        self.catw[i] = np.asarray(w, dtype=np.float64).copy()

    def setCategoryRates(self, r):
        """CPU/BeagleCPUImpl.hpp:770-779 (rates kept in double, index 0)."""
        self.rates[0] = np.asarray(r, dtype=np.float64).copy()

    def setCategoryRatesWithIndex(self, i, r):
        self.rates[i] = np.asarray(r, dtype=np.float64).copy()

    def setPatternWeights(self, w):
        self.patw = np.asarray(w, dtype=np.float64).copy()

    # ---- transition matrices ----------------------------------------------
    def updateTransitionMatrices(self, e, probIdx, d1Idx, d2Idx, t, rates=None):
        """CPU/EigenDecompositionCube.hpp:105-322.

        P[c][i][j] = max(0, sum_k C[i][j][k] exp(lambda_k * t * r_c)), pad column 1;
        D1 = sum_k C[i][j][k] lambda_k r_c exp(..), D2 likewise with (lambda_k r_c)^2,
        pad column 0 for both (no clamp on derivatives)."""
        count = len(probIdx)
        r = self.rates[0] if rates is None else rates
        lam = self.evals[e]
        cube = self.cube[e]
        for u in range(count):
            for c in range(self.C):
                ex = np.exp(lam * (t[u] * r[c]))
                P = cube @ ex
                self.matrices[probIdx[u]][c, :, :self.S] = np.where(P > 0, P, 0.0)
                self.matrices[probIdx[u]][c, :, self.S] = 1.0
                if d1Idx is not None:
                    sl = lam * r[c]
                    self.matrices[d1Idx[u]][c, :, :self.S] = cube @ (sl * ex)
                    self.matrices[d1Idx[u]][c, :, self.S] = 0.0
                    if d2Idx is not None:
                        self.matrices[d2Idx[u]][c, :, :self.S] = cube @ (sl * sl * ex)
                        self.matrices[d2Idx[u]][c, :, self.S] = 0.0

    def updateTransitionMatricesWithMultipleModels(self, eig, rix, probIdx, d1Idx, d2Idx, t):
        """CPU/BeagleCPUImpl.hpp:1256-1289: matrix u from eigen system eig[u]
        and category rates rix[u] (updateTransitionMatrices one at a time)."""
        for u in range(len(probIdx)):
            self.updateTransitionMatrices(
                eig[u], [probIdx[u]], None if d1Idx is None else [d1Idx[u]],
                None if (d1Idx is None or d2Idx is None) else [d2Idx[u]], [t[u]],
                rates=self.rates[rix[u]])

    def updateTransitionMatricesWithModelCategories(self, eig, probIdx, d1Idx, d2Idx, t):
        """CPU/EigenDecompositionCube.hpp:326-470: category c of every matrix
        from eigen system eig[c], exp(lambda t) with no category rate; pad
        column 1 for P, 0 for the derivatives."""
        for u in range(len(probIdx)):
            for c in range(self.C):
                lam, cube = self.evals[eig[c]], self.cube[eig[c]]
                ex = np.exp(lam * t[u])
                P = cube @ ex
                self.matrices[probIdx[u]][c, :, :self.S] = np.where(P > 0, P, 0.0)
                self.matrices[probIdx[u]][c, :, self.S] = 1.0
                if d1Idx is not None:
                    self.matrices[d1Idx[u]][c, :, :self.S] = cube @ (lam * ex)
                    self.matrices[d1Idx[u]][c, :, self.S] = 0.0
                    if d2Idx is not None:
                        self.matrices[d2Idx[u]][c, :, :self.S] = cube @ (lam * lam * ex)
                        self.matrices[d2Idx[u]][c, :, self.S] = 0.0

    def setTransitionMatrix(self, m, mat, padded):
        """CPU/BeagleCPUImpl.hpp:1035-1054: [C][S][S] in, pad column = paddedValue."""
        self.matrices[m][:, :, :self.S] = np.asarray(mat, dtype=np.float64).reshape(
            self.C, self.S, self.S)
        self.matrices[m][:, :, self.S] = padded

    def getTransitionMatrix(self, m):
        return self.matrices[m][:, :, :self.S].reshape(-1).copy()

    def transposeTransitionMatrices(self, inIdx, outIdx):
        """CPU/BeagleCPUImpl.hpp:1175-1222 (the pad column is left as it was)."""
        for a, b in zip(inIdx, outIdx):
            self.matrices[b][:, :, :self.S] = np.transpose(
                self.matrices[a][:, :, :self.S], (0, 2, 1))

    def convolveTransitionMatrices(self, first, second, result):
        """CPU/BeagleCPUImpl.hpp:1096-1160: C = A @ B per category, pad column 1."""
        for a, b, r in zip(first, second, result):
            if a == r or b == r:
                return ERROR_OUT_OF_RANGE
            self.matrices[r][:, :, :self.S] = (self.matrices[a][:, :, :self.S]
                                               @ self.matrices[b][:, :, :self.S])
            self.matrices[r][:, :, self.S] = 1.0
        return SUCCESS

    # ---- partials ----------------------------------------------------------
    def _child(self, idx, mat):
        """Per-category product P . x for one child (tip states or partials).

        Tip states select column `state` of P, the missing state S selecting the
        pad column (CPU/BeagleCPUImpl.hpp:4226-4258, 4300-4352, 4469-4524)."""
        M = self.matrices[mat]
        if self.states[idx] is not None:
            st = self.states[idx]
            return np.transpose(M[:, :, st], (0, 2, 1))          # [c][p][i]
        x = self.partials[idx]
        return np.einsum('cij,cpj->cpi', M[:, :, :self.S], x)

    def _rescale(self, dest, scale_idx, cumulative):
        """CPU/BeagleCPUImpl.hpp:4008-4056: per pattern max over categories and
        states (0 -> 1), multiply by 1/max, store log(max) (LOG) or max (RAW),
        add log(max) to the cumulative buffer when one is given."""
        mx = dest.max(axis=(0, 2))
        mx = np.where(mx == 0, 1.0, mx)
        dest *= (1.0 / mx)[None, :, None]
        lg = np.log(mx)
        self.scale[scale_idx][:] = lg if self.log_scalers else mx
        if cumulative is not None:
            cumulative += lg

    def updatePartials(self, ops, cumulativeScaleIndex=OP_NONE):
        """CPU/BeagleCPUImpl.hpp:1497-1686 (manual scaling): for each 7-int op
        (dest, writeScale, readScale, child1, mat1, child2, mat2) compute
        dest = (P1 . x1) * (P2 . x2); then rescale when writeScale >= 0, or divide
        by the stored factor when only readScale >= 0 (FixedScaling variants)."""
        ops = np.asarray(ops, dtype=np.int64).reshape(-1, 7)
        cum = self.scale[cumulativeScaleIndex] if cumulativeScaleIndex != OP_NONE else None
        for dest, wsc, rsc, c1, m1, c2, m2 in ops:
            out = self._child(c1, m1) * self._child(c2, m2)
            if wsc >= 0:
                self._rescale(out, wsc, cum)
            elif rsc >= 0:
                out *= (1.0 / self.scale[rsc])[None, :, None]
            self.partials[dest] = out

    def updatePrePartials(self, ops, cumulativeScaleIndex=OP_NONE):
        """CPU/BeagleCPUImpl.hpp:1689-1862 with calcPrePartialsPartials/States
        (:4530-4662): op = (dest, writeScale, readScale, parentPre, P_node,
        sibling, P_sibling);
        dest[c,p,j] = sum_i P_node[c][i][j] * pre[c,p,i] * (P_sib . x_sib)[c,p,i].
        Rescaling never touches a cumulative buffer (:1694-1696)."""
        ops = np.asarray(ops, dtype=np.int64).reshape(-1, 7)
        for dest, wsc, rsc, par, m1, sib, m2 in ops:
            z = self.partials[par] * self._child(sib, m2)
            M = self.matrices[m1][:, :, :self.S]
            out = np.einsum('cij,cpi->cpj', M, z)
            if wsc >= 0:
                self._rescale(out, wsc, None)
            self.partials[dest] = out

    # ---- partitions ---------------------------------------------------------
    def setPatternPartitions(self, n, parts):
        """CPU/BeagleCPUImpl.hpp:803-920 for contiguous, ascending partitions
        (the reference reorders patterns otherwise): start pattern of each."""
        parts = np.asarray(parts, dtype=np.int64)
        assert parts[0] == 0 and np.all(np.diff(parts) >= 0) and parts[-1] == n - 1
        self.part_start = np.searchsorted(parts, np.arange(n + 1), side='left')
        self.part_start[n] = self.P

    def _range(self, part):
        return slice(int(self.part_start[part]), int(self.part_start[part + 1]))

    def _rescale_range(self, out, rng, scale_idx, cumulative):
        """rescalePartialsByPartition (CPU/BeagleCPUImpl.hpp:4060-4110): the
        rescaling of _rescale restricted to the partition's patterns."""
        mx = out.max(axis=(0, 2))
        mx = np.where(mx == 0, 1.0, mx)
        out *= (1.0 / mx)[None, :, None]
        lg = np.log(mx)
        self.scale[scale_idx][rng] = lg if self.log_scalers else mx
        if cumulative is not None:
            cumulative[rng] += lg

    def updatePartialsByPartition(self, ops):
        """upPartials with byPartition (CPU/BeagleCPUImpl.hpp:1497-1686): 9-int ops,
        field 7 the partition, field 8 its cumulative scale index; only the
        partition's patterns of dest are computed."""
        ops = np.asarray(ops, dtype=np.int64).reshape(-1, 9)
        for dest, wsc, rsc, c1, m1, c2, m2, part, cidx in ops:
            rng = self._range(part)
            out = (self._child(c1, m1) * self._child(c2, m2))[:, rng, :]
            cum = self.scale[cidx] if cidx != OP_NONE else None
            if wsc >= 0:
                self._rescale_range(out, rng, wsc, cum)
            elif rsc >= 0:
                out *= (1.0 / self.scale[rsc][rng])[None, :, None]
            self.partials[dest][:, rng, :] = out

    def updatePrePartialsByPartition(self, ops):
        """upPrePartials with byPartition (CPU/BeagleCPUImpl.hpp:1689-1862)."""
        ops = np.asarray(ops, dtype=np.int64).reshape(-1, 9)
        for dest, wsc, rsc, par, m1, sib, m2, part, cidx in ops:
            rng = self._range(part)
            z = (self.partials[par] * self._child(sib, m2))[:, rng, :]
            M = self.matrices[m1][:, :, :self.S]
            out = np.einsum('cij,cpi->cpj', M, z)
            if wsc >= 0:
                self._rescale_range(out, rng, wsc, None)
            self.partials[dest][:, rng, :] = out

    def resetScaleFactorsByPartition(self, idx, part):
        """CPU/BeagleCPUImpl.hpp:2885-2900."""
        self.scale[idx][self._range(part)] = 0.0

    def accumulateScaleFactorsByPartition(self, idxs, cumulative, part):
        """CPU/BeagleCPUImpl.hpp:2804-2828."""
        rng = self._range(part)
        for i in idxs:
            s = self.scale[i][rng]
            self.scale[cumulative][rng] += s if self.log_scalers else np.log(s)

    def removeScaleFactorsByPartition(self, idxs, cumulative, part):
        """CPU/BeagleCPUImpl.hpp:2850-2870."""
        rng = self._range(part)
        for i in idxs:
            s = self.scale[i][rng]
            self.scale[cumulative][rng] -= s if self.log_scalers else np.log(s)

    def calculateRootLogLikelihoodsByPartition(self, bufs, cws, sfs, cums, parts):
        """CPU/BeagleCPUImpl.hpp:2349-2388 (count 1): per partition i the lnL of
        root bufs[i] over partition parts[i]'s patterns; and their total."""
        if not hasattr(self, 'site_lnl') or self.site_lnl is None:
            self.site_lnl = np.zeros(self.P)
        byp = []
        for buf, cw, sf, cum, part in zip(bufs, cws, sfs, cums, parts):
            rng = self._range(part)
            root = self.partials[buf][:, rng, :]
            integ = np.einsum('c,cpi->pi', self.catw[cw], root)
            site = np.log(integ @ self.freqs[sf])
            if cum != OP_NONE:
                site = site + self.scale[cum][rng]
            self.site_lnl[rng] = site
            byp.append(float(np.dot(site, self.patw[rng])))
        return np.array(byp), float(sum(byp))

    # ---- scale factors -----------------------------------------------------
    def resetScaleFactors(self, idx):
        """CPU/BeagleCPUImpl.hpp:2874-2883."""
        self.scale[idx][:] = 0.0

    def accumulateScaleFactors(self, idxs, cumulative):
        """CPU/BeagleCPUImpl.hpp:2763-2801 (log of RAW scalers)."""
        for i in idxs:
            s = self.scale[i]
            self.scale[cumulative] += s if self.log_scalers else np.log(s)

    def removeScaleFactors(self, idxs, cumulative):
        """CPU/BeagleCPUImpl.hpp:2830-2846."""
        for i in idxs:
            s = self.scale[i]
            self.scale[cumulative] -= s if self.log_scalers else np.log(s)

    def copyScaleFactors(self, dst, src):
        self.scale[dst][:] = self.scale[src]

    def getScaleFactors(self, idx):
        return self.scale[idx].copy()

    # ---- reductions -----------------------------------------------------------
    def calculateRootLogLikelihoods(self, bufs, cws, sfs, cums):
        """CPU/BeagleCPUImpl.hpp:2630-2691 (one root, index lists of length 1 as
        in the C call): site lnL = log(sum_i pi_i sum_c w_c root[c,p,i]) +
        cumulative[p]; returns sum_p W_p * site lnL."""
        buf, cw, sf, cum = bufs[0], cws[0], sfs[0], cums[0]
        root = self.partials[buf]
        integ = np.einsum('c,cpi->pi', self.catw[cw], root)
        site = np.log(integ @ self.freqs[sf])
        if cum != OP_NONE:
            site = site + self.scale[cum]
        self.site_lnl = site
        return float(np.dot(site, self.patw))

    def getSiteLogLikelihoods(self):
        return self.site_lnl.copy()

    def calculateEdgeDerivatives(self, post, pre, dmat, cw, per_site=True, sums=True,
                                 sumsq=True):
        """CPU/BeagleCPUImpl.hpp:1940-2083, 2086-2119, 2240-2285.

        Per branch b and pattern p:
          num = sum_c w_c sum_k pre[c,p,k] (D_c . post)[c,p,k]
          den = sum_c w_c sum_k pre[c,p,k] post[c,p,k]
        d = num/den; returns (per-site d [count][P], sum_p W_p d, sum_p W_p d^2).
        Category weights come from categoryWeightsIndices[0] only.

        Compact (tip-state) post buffers use D[c][k][state] for the numerator and
        pre[state] for the denominator.  A missing state (S) there is handled as
        an all-ones partial (den = sum_k pre[k], num = sum_k pre[k] D[k][pad]);
        the reference instead reads pre[state % S] (:2106-2108, marked TODO in
        the reference), so inputs with missing tip states should use tip
        partials when compared against the compiled reference."""
        w = self.catw[cw[0]]
        n = len(post)
        per_site = np.zeros((n, self.P))
        for b in range(n):
            D = self.matrices[dmat[b]]
            prb = self.partials[pre[b]]
            if self.states[post[b]] is not None:
                st = self.states[post[b]]
                numc = np.einsum('ckp,cpk->cp', D[:, :, st], prb)
                sel = np.where(st < self.S, st, 0)
                denc = np.take_along_axis(prb, sel[None, :, None], axis=2)[:, :, 0]
                miss = st >= self.S
                if miss.any():
                    denc[:, miss] = prb[:, miss, :].sum(axis=2)
            else:
                x = self.partials[post[b]]
                y = np.einsum('ckj,cpj->cpk', D[:, :, :self.S], x)
                numc = (prb * y).sum(axis=2)
                denc = (prb * x).sum(axis=2)
            num = w @ numc
            den = w @ denc
            per_site[b] = num / den
        self.site_d1 = per_site[-1].copy() if n else self.site_d1
        sums = per_site @ self.patw
        sumsq = (per_site * per_site) @ self.patw
        return per_site, sums, sumsq

    def calculateCrossProductDerivative(self, post, pre, crates, cw, lengths, out):
        """CPU/BeagleCPUImpl.hpp:1865-1937 (calcCrossProducts), :2122-2237
        (calcCrossProductsStates / calcCrossProductsPartials); the 4-state
        forms (CPU/BeagleCPU4StateImpl.hpp:1088-1251) compute the same sums.

        For every listed branch b and pattern p, with w = category weights
        [cw[0]], r = category rates [crates[0]] and t = lengths[b]:
          den = sum_c w_c sum_k pre[c,p,k] post[c,p,k]
          out[k][j] += W_p / den * sum_c w_c r_c t pre[c,p,k] post[c,p,j]
        A compact (tip-state) post buffer is its one-hot row, all ones for the
        missing state.  `out` (S x S, row-major, the caller's array) is added
        to, not cleared, as in the reference; sums of squares are not
        computed there either."""
        w = self.catw[cw[0]]
        r = self.rates[crates[0]]
        S = self.S
        acc = np.zeros((S, S))
        for b in range(len(post)):
            prb = self.partials[pre[b]]                         # [C][P][S]
            if self.states[post[b]] is not None:
                st = self.states[post[b]]
                x = np.zeros_like(prb)
                ok = st < S
                x[:, np.where(ok)[0], st[ok]] = 1.0
                x[:, ~ok, :] = 1.0
            else:
                x = self.partials[post[b]]
            den = np.einsum('c,cpk,cpk->p', w, prb, x)
            coef = self.patw / den
            acc += np.einsum('c,p,cpk,cpj->kj', w * r * lengths[b], coef, prb, x)
        out = np.asarray(out)
        out += acc.reshape(out.shape)
        return out

    def calculateEdgeLogLikelihoods(self, parent, child, prob, d1, d2, cw, sf, cum):
        """CPU/BeagleCPUImpl.hpp:3209-3322, 3753-3994: for one edge,
        L[c,p,i] = parent[c,p,i] * (P . child)[c,p,i];
        site lnL = log(sum_i pi_i sum_c w_c L) + cumulative[p]; with derivative
        matrices, d1 = E[P']/L and d2 = E[P'']/L - d1^2 per site.
        Returns (code, lnL, sum d1 or None, sum d2 or None)."""
        par = self.partials[parent]
        f = self.freqs[sf]
        w = self.catw[cw]

        def integ(mat):
            y = self._child(child, mat)
            return np.einsum('c,cpi,i->p', w, par * y, f)

        L = integ(prob)
        site = np.log(L)
        if cum != OP_NONE:
            site = site + self.scale[cum]
        self.site_lnl = site
        total = float(np.dot(site, self.patw))
        s1 = s2 = None
        if d1 is not None:
            g1 = integ(d1) / L
            self.site_d1 = g1
            s1 = float(np.dot(g1, self.patw))
            if d2 is not None:
                g2 = integ(d2) / L - g1 * g1
                self.site_d2 = g2
                s2 = float(np.dot(g2, self.patw))
        code = ERROR_FLOATING_POINT if total != total else SUCCESS
        return code, total, s1, s2

    def calculateEdgeLogLikelihoodsByPartition(self, parents, children, probs, d1s, d2s, cws,
                                               sfs, cums, parts):
        """CPU/BeagleCPUImpl.hpp:3008-3110 with :3325-3450 and :3452-3587
        (count 1): for entry i, the edge lnL of (parents[i], children[i],
        probs[i]) over partition parts[i]'s patterns, with the site values of
        calculateEdgeLogLikelihoods written for those patterns; with both
        derivative lists, also the d1 and d2 sums (d1 alone is
        NO_IMPLEMENTATION there).  Returns (code, lnL by entry, lnL, d1 by
        entry, d1, d2 by entry, d2)."""
        if d1s is not None and d2s is None:
            return ERROR_NO_IMPLEMENTATION, None, None, None, None, None, None
        derivs = d1s is not None
        for name in ('site_lnl', 'site_d1', 'site_d2'):
            if getattr(self, name, None) is None:
                setattr(self, name, np.zeros(self.P))
        byp, d1p, d2p = [], [], []
        for i, part in enumerate(parts):
            rng = self._range(part)
            par = self.partials[parents[i]][:, rng, :]
            f = self.freqs[sfs[i]]
            w = self.catw[cws[i]]

            def integ(mat):
                y = self._child(children[i], mat)[:, rng, :]
                return np.einsum('c,cpi,i->p', w, par * y, f)

            L = integ(probs[i])
            site = np.log(L)
            if cums[i] != OP_NONE:
                site = site + self.scale[cums[i]][rng]
            self.site_lnl[rng] = site
            byp.append(float(np.dot(site, self.patw[rng])))
            if derivs:
                g1 = integ(d1s[i]) / L
                g2 = integ(d2s[i]) / L - g1 * g1
                self.site_d1[rng] = g1
                self.site_d2[rng] = g2
                d1p.append(float(np.dot(g1, self.patw[rng])))
                d2p.append(float(np.dot(g2, self.patw[rng])))
        total = float(sum(byp))
        code = ERROR_FLOATING_POINT if total != total else SUCCESS
        if not derivs:
            return code, np.array(byp), total, None, None, None, None
        t1, t2 = float(sum(d1p)), float(sum(d2p))
        if t1 != t1 or t2 != t2:
            code = ERROR_FLOATING_POINT
        return code, np.array(byp), total, np.array(d1p), t1, np.array(d2p), t2
