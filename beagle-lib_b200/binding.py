"""ctypes binding of a BEAGLE-style C API.

The same table binds two libraries that share one calling convention:

* ``libbeagle_b200.so`` -- this package's C-ABI (``include/beagle_b200.h``),
  whose entry points are the ``beagle.h`` calls renamed ``beagleB200*``;
* a stock ``libhmsbeagle.so`` (``beagle*`` names, ``libhmsbeagle/beagle.h``),
  which the test-suite uses to run the reference CPU implementation.

Arguments are numpy arrays (converted to contiguous float64 / int32) or plain
Python numbers; every call returns the library's ``int`` code and raises
``BeagleError`` on a negative one unless ``check=False`` is passed.
"""

import ctypes
import numpy as np

_i = ctypes.c_int
_l = ctypes.c_long
_d = ctypes.c_double
_p = ctypes.c_void_p

# name -> argtypes (all return int unless listed in _RESTYPES)
_SIGS = {
    "BeginCapture": [_i], "EndCapture": [_i, _p], "LaunchGraph": [_i, _i],
    "LaunchGraphWithLengths": [_i, _i, _p, _i],
    "FinalizeInstance": [_i],
    "Finalize": [],
    "SetCPUThreadCount": [_i, _i],
    "SetTipStates": [_i, _i, _p],
    "SetTipPartials": [_i, _i, _p],
    "SetPartials": [_i, _i, _p],
    "GetPartials": [_i, _i, _i, _p],
    "SetRootPrePartials": [_i, _p, _p, _i],
    "SetEigenDecomposition": [_i, _i, _p, _p, _p],
    "SetStateFrequencies": [_i, _i, _p],
    "SetCategoryWeights": [_i, _i, _p],
    "SetCategoryRates": [_i, _p],
    "SetCategoryRatesWithIndex": [_i, _i, _p],
    "SetPatternWeights": [_i, _p],
    "SetPatternPartitions": [_i, _i, _p],
    "ConvolveTransitionMatrices": [_i, _p, _p, _p, _i],
    "AddTransitionMatrices": [_i, _p, _p, _p, _i],
    "TransposeTransitionMatrices": [_i, _p, _p, _i],
    "UpdateTransitionMatrices": [_i, _i, _p, _p, _p, _p, _i],
    "UpdateTransitionMatricesWithModelCategories": [_i, _p, _p, _p, _p, _p, _i],
    "UpdateTransitionMatricesWithMultipleModels": [_i, _p, _p, _p, _p, _p, _p, _i],
    "SetTransitionMatrix": [_i, _i, _p, _d],
    "SetDifferentialMatrix": [_i, _i, _p],
    "GetTransitionMatrix": [_i, _i, _p],
    "SetTransitionMatrices": [_i, _p, _p, _p, _i],
    "UpdatePartials": [_i, _p, _i, _i],
    "UpdatePrePartials": [_i, _p, _i, _i],
    "UpdatePartialsByPartition": [_i, _p, _i],
    "UpdatePrePartialsByPartition": [_i, _p, _i],
    "WaitForPartials": [_i, _p, _i],
    "AccumulateScaleFactors": [_i, _p, _i, _i],
    "AccumulateScaleFactorsByPartition": [_i, _p, _i, _i, _i],
    "RemoveScaleFactors": [_i, _p, _i, _i],
    "RemoveScaleFactorsByPartition": [_i, _p, _i, _i, _i],
    "ResetScaleFactors": [_i, _i],
    "ResetScaleFactorsByPartition": [_i, _i, _i],
    "CopyScaleFactors": [_i, _i, _i],
    "GetScaleFactors": [_i, _i, _p],
    "CalculateRootLogLikelihoods": [_i, _p, _p, _p, _p, _i, _p],
    "CalculateRootLogLikelihoodsByPartition": [_i, _p, _p, _p, _p, _p, _i, _i, _p, _p],
    "CalculateEdgeDerivatives": [_i, _p, _p, _p, _p, _i, _p, _p, _p],
    "UpdatePrePartialsWithDerivatives": [_i, _p, _i, _p, _p, _p, _p, _p],
    "UpdatePartialsWithRootLogLikelihood": [_i, _p, _i, _i, _i, _i, _i, _p],
    "GetTunedVariants": [_i, _p],
    "CalculateCrossProductDerivative": [_i, _p, _p, _p, _p, _p, _i, _p, _p],
    "CalculateEdgeLogLikelihoods": [_i, _p, _p, _p, _p, _p, _p, _p, _p, _i, _p, _p, _p],
    "CalculateEdgeLogLikelihoodsByPartition": [_i] + [_p] * 9 + [_i, _i] + [_p] * 6,
    "GetLogLikelihood": [_i, _p],
    "GetDerivatives": [_i, _p, _p],
    "GetSiteLogLikelihoods": [_i, _p],
    "GetSiteDerivatives": [_i, _p, _p],
    "GetCudaStream": [_i, _p],
    "InjectKernelTimeout": [_i, _i],
}

ERRORS = {
    -1: "BEAGLE_ERROR_GENERAL", -2: "BEAGLE_ERROR_OUT_OF_MEMORY",
    -3: "BEAGLE_ERROR_UNIDENTIFIED_EXCEPTION", -4: "BEAGLE_ERROR_UNINITIALIZED_INSTANCE",
    -5: "BEAGLE_ERROR_OUT_OF_RANGE", -6: "BEAGLE_ERROR_NO_RESOURCE",
    -7: "BEAGLE_ERROR_NO_IMPLEMENTATION", -8: "BEAGLE_ERROR_FLOATING_POINT",
}


class BeagleError(RuntimeError):
    def __init__(self, call, code):
        super().__init__(f"{call} returned {code} ({ERRORS.get(code, 'unknown')})")
        self.code = code


class InstanceDetails(ctypes.Structure):
    """Layout of ``BeagleInstanceDetails`` (libhmsbeagle/beagle.h:216-226)."""
    _fields_ = [("resourceNumber", _i), ("resourceName", ctypes.c_char_p),
                ("implName", ctypes.c_char_p), ("implDescription", ctypes.c_char_p),
                ("flags", _l)]


class Resource(ctypes.Structure):
    """Layout of ``BeagleResource`` (libhmsbeagle/beagle.h:231-236)."""
    _fields_ = [("name", ctypes.c_char_p), ("description", ctypes.c_char_p),
                ("supportFlags", _l), ("requiredFlags", _l)]


class ResourceList(ctypes.Structure):
    _fields_ = [("list", ctypes.POINTER(Resource)), ("length", _i)]


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_p)


class BeagleLib:
    """A loaded BEAGLE-style library, with symbols ``<prefix><Name>``."""

    def __init__(self, path, prefix, mode=ctypes.RTLD_GLOBAL):
        self.path = path
        self.prefix = prefix
        self.lib = ctypes.CDLL(path, mode=mode)
        self.fn = {}
        for name, args in _SIGS.items():
            f = getattr(self.lib, prefix + name, None)
            if f is None:
                continue
            f.argtypes = args
            f.restype = _i
            self.fn[name] = f
        ci = getattr(self.lib, prefix + "CreateInstance")
        ci.argtypes = [_i] * 9 + [_p, _i, _l, _l, ctypes.POINTER(InstanceDetails)]
        ci.restype = _i
        self.fn["CreateInstance"] = ci
        rl = getattr(self.lib, prefix + "GetResourceList")
        rl.argtypes = []
        rl.restype = ctypes.POINTER(ResourceList)
        self.fn["GetResourceList"] = rl

    def resources(self):
        rl = self.fn["GetResourceList"]().contents
        return [(rl.list[i].name.decode(), rl.list[i].supportFlags, rl.list[i].requiredFlags)
                for i in range(rl.length)]

    def create(self, tipCount, partialsBufferCount, compactBufferCount, stateCount,
               patternCount, eigenBufferCount, matrixBufferCount, categoryCount,
               scaleBufferCount, resources=None, preferenceFlags=0, requirementFlags=0):
        info = InstanceDetails()
        res = None if resources is None else _i32(resources)
        nres = 0 if resources is None else len(resources)
        h = self.fn["CreateInstance"](tipCount, partialsBufferCount, compactBufferCount,
                                      stateCount, patternCount, eigenBufferCount,
                                      matrixBufferCount, categoryCount, scaleBufferCount,
                                      _ptr(res), nres, preferenceFlags, requirementFlags,
                                      ctypes.byref(info))
        if h < 0:
            raise BeagleError(self.prefix + "CreateInstance", h)
        return Instance(self, h, info, dict(
            tipCount=tipCount, bufferCount=partialsBufferCount + compactBufferCount,
            stateCount=stateCount, patternCount=patternCount,
            categoryCount=categoryCount))


class Instance:
    """One instance of a BeagleLib; methods mirror the beagle.h calls."""

    def __init__(self, blib, handle, info, dims):
        self.blib = blib
        self.h = handle
        self.info = info
        self.impl_name = info.implName.decode() if info.implName else ""
        self.flags = info.flags
        self._keep = []           # output arrays an ASYNCH instance fills at its next sync
        self._graph_keep = []     # ... and those a captured graph fills at every launch
        self._capturing = False
        self.__dict__.update(dims)

    def _call(self, name, *args, check=True):
        code = self.blib.fn[name](self.h, *args)
        if check and code < 0:
            raise BeagleError(self.blib.prefix + name, code)
        return code

    def __del__(self):
        try:
            self.finalize()
        except Exception:
            pass

    # CUDA graphs (ASYNCH instances)
    def beginCapture(self):
        code = self._call("BeginCapture")
        self._capturing = True
        return code

    def endCapture(self):
        g = np.full(1, -1, dtype=np.int32)
        self._capturing = False
        self._call("EndCapture", _ptr(g))
        return int(g[0])

    def launchGraph(self, graph):
        return self._call("LaunchGraph", graph)

    def launchGraphWithLengths(self, graph, lengths):
        """Launch a graph whose captured matrix updates read new branch
        lengths (all of them, in capture order)."""
        t = _f64(lengths)
        return self._call("LaunchGraphWithLengths", graph, _ptr(t), t.size)

    def finalize(self):
        if self.h is not None and self.h >= 0:
            self._call("FinalizeInstance")
            self.h = None
            self._keep = []

    # data in
    def setCPUThreadCount(self, n):
        return self._call("SetCPUThreadCount", n)

    def setTipStates(self, tip, states):
        a = _i32(states)
        return self._call("SetTipStates", tip, _ptr(a))

    def setTipPartials(self, tip, partials):
        a = _f64(partials)
        return self._call("SetTipPartials", tip, _ptr(a))

    def setPartials(self, buf, partials):
        a = _f64(partials)
        return self._call("SetPartials", buf, _ptr(a))

    def getPartials(self, buf, scaleIndex=-1):
        out = np.zeros(self.categoryCount * self.patternCount * self.stateCount)
        self._call("GetPartials", buf, scaleIndex, _ptr(out))
        return out

    def setRootPrePartials(self, bufs, freqIdx, check=True):
        b, f = _i32(bufs), _i32(freqIdx)
        return self._call("SetRootPrePartials", _ptr(b), _ptr(f), len(b), check=check)

    def setEigenDecomposition(self, e, evec, ivec, evals):
        a, b, c = _f64(evec), _f64(ivec), _f64(evals)
        return self._call("SetEigenDecomposition", e, _ptr(a), _ptr(b), _ptr(c))

    def setStateFrequencies(self, i, f):
        a = _f64(f)
        return self._call("SetStateFrequencies", i, _ptr(a))

    def setCategoryWeights(self, i, w):
        a = _f64(w)
        return self._call("SetCategoryWeights", i, _ptr(a))

    def setCategoryRates(self, r):
        a = _f64(r)
        return self._call("SetCategoryRates", _ptr(a))

    def setCategoryRatesWithIndex(self, i, r):
        a = _f64(r)
        return self._call("SetCategoryRatesWithIndex", i, _ptr(a))

    def setPatternWeights(self, w):
        a = _f64(w)
        return self._call("SetPatternWeights", _ptr(a))

    def setPatternPartitions(self, n, parts):
        a = _i32(parts)
        return self._call("SetPatternPartitions", n, _ptr(a))

    # matrices
    def updateTransitionMatrices(self, e, probIdx, d1Idx, d2Idx, lengths):
        p = _i32(probIdx)
        d1 = None if d1Idx is None else _i32(d1Idx)
        d2 = None if d2Idx is None else _i32(d2Idx)
        t = _f64(lengths)
        return self._call("UpdateTransitionMatrices", e, _ptr(p), _ptr(d1), _ptr(d2),
                          _ptr(t), len(p))

    def updateTransitionMatricesWithMultipleModels(self, eig, rateIdx, probIdx, d1Idx,
                                                   d2Idx, lengths):
        e, r, p = _i32(eig), _i32(rateIdx), _i32(probIdx)
        d1 = None if d1Idx is None else _i32(d1Idx)
        d2 = None if d2Idx is None else _i32(d2Idx)
        t = _f64(lengths)
        return self._call("UpdateTransitionMatricesWithMultipleModels", _ptr(e), _ptr(r),
                          _ptr(p), _ptr(d1), _ptr(d2), _ptr(t), len(p))

    def updateTransitionMatricesWithModelCategories(self, eig, probIdx, d1Idx, d2Idx,
                                                    lengths):
        e, p = _i32(eig), _i32(probIdx)
        d1 = None if d1Idx is None else _i32(d1Idx)
        d2 = None if d2Idx is None else _i32(d2Idx)
        t = _f64(lengths)
        return self._call("UpdateTransitionMatricesWithModelCategories", _ptr(e), _ptr(p),
                          _ptr(d1), _ptr(d2), _ptr(t), len(p))

    def setTransitionMatrix(self, m, mat, padded=1.0):
        a = _f64(mat)
        return self._call("SetTransitionMatrix", m, _ptr(a), float(padded))

    def setDifferentialMatrix(self, m, mat):
        a = _f64(mat)
        return self._call("SetDifferentialMatrix", m, _ptr(a))

    def setTransitionMatrices(self, idx, mats, pads):
        i, m, p = _i32(idx), _f64(mats), _f64(pads)
        return self._call("SetTransitionMatrices", _ptr(i), _ptr(m), _ptr(p), len(i))

    def getTransitionMatrix(self, m):
        out = np.zeros(self.categoryCount * self.stateCount * self.stateCount)
        self._call("GetTransitionMatrix", m, _ptr(out))
        return out

    def transposeTransitionMatrices(self, inIdx, outIdx, check=True):
        a, b = _i32(inIdx), _i32(outIdx)
        return self._call("TransposeTransitionMatrices", _ptr(a), _ptr(b), len(a),
                          check=check)

    def convolveTransitionMatrices(self, first, second, result, check=True):
        a, b, c = _i32(first), _i32(second), _i32(result)
        return self._call("ConvolveTransitionMatrices", _ptr(a), _ptr(b), _ptr(c), len(a),
                          check=check)

    # partials
    def updatePartials(self, ops, cumulativeScaleIndex=-1, check=True):
        a = _i32(ops).reshape(-1)
        return self._call("UpdatePartials", _ptr(a), len(a) // 7, cumulativeScaleIndex,
                          check=check)

    def updatePrePartials(self, ops, cumulativeScaleIndex=-1, check=True):
        a = _i32(ops).reshape(-1)
        return self._call("UpdatePrePartials", _ptr(a), len(a) // 7, cumulativeScaleIndex,
                          check=check)

    def updatePartialsByPartition(self, ops, check=True):
        a = _i32(ops).reshape(-1)
        return self._call("UpdatePartialsByPartition", _ptr(a), len(a) // 9, check=check)

    def updatePrePartialsByPartition(self, ops, check=True):
        a = _i32(ops).reshape(-1)
        return self._call("UpdatePrePartialsByPartition", _ptr(a), len(a) // 9, check=check)

    def waitForPartials(self, bufs):
        a = _i32(bufs)
        code = self._call("WaitForPartials", _ptr(a), len(a))
        self._keep = []
        return code

    # scale factors
    def resetScaleFactors(self, idx):
        return self._call("ResetScaleFactors", idx)

    def resetScaleFactorsByPartition(self, idx, part):
        return self._call("ResetScaleFactorsByPartition", idx, part)

    def accumulateScaleFactors(self, idxs, cumulative):
        a = _i32(idxs)
        return self._call("AccumulateScaleFactors", _ptr(a), len(a), cumulative)

    def accumulateScaleFactorsByPartition(self, idxs, cumulative, part):
        a = _i32(idxs)
        return self._call("AccumulateScaleFactorsByPartition", _ptr(a), len(a), cumulative,
                          part)

    def removeScaleFactors(self, idxs, cumulative):
        a = _i32(idxs)
        return self._call("RemoveScaleFactors", _ptr(a), len(a), cumulative)

    def removeScaleFactorsByPartition(self, idxs, cumulative, part):
        a = _i32(idxs)
        return self._call("RemoveScaleFactorsByPartition", _ptr(a), len(a), cumulative, part)

    def copyScaleFactors(self, dst, src):
        return self._call("CopyScaleFactors", dst, src)

    def getScaleFactors(self, idx):
        out = np.zeros(self.patternCount)
        self._call("GetScaleFactors", idx, _ptr(out))
        return out

    # reductions
    def calculateRootLogLikelihoods(self, bufs, cw, sf, cum, check=True):
        b, w, f, c = _i32(bufs), _i32(cw), _i32(sf), _i32(cum)
        out = np.zeros(1)
        code = self._call("CalculateRootLogLikelihoods", _ptr(b), _ptr(w), _ptr(f), _ptr(c),
                          len(b), _ptr(out), check=check)
        return (code, float(out[0])) if not check else float(out[0])

    def calculateRootLogLikelihoodsByPartition(self, bufs, cw, sf, cum, parts):
        b, w, f, c, p = _i32(bufs), _i32(cw), _i32(sf), _i32(cum), _i32(parts)
        byp = np.zeros(len(p))
        tot = np.zeros(1)
        self._call("CalculateRootLogLikelihoodsByPartition", _ptr(b), _ptr(w), _ptr(f),
                   _ptr(c), _ptr(p), len(p), 1, _ptr(byp), _ptr(tot))
        return byp, float(tot[0])

    def calculateEdgeDerivatives(self, post, pre, dmat, cw, per_site=True, sums=True,
                                 sumsq=True, check=True):
        a, b, d, w = _i32(post), _i32(pre), _i32(dmat), _i32(cw)
        n = len(a)
        o1 = np.zeros(n * self.patternCount) if per_site else None
        o2 = np.zeros(n) if sums else None
        o3 = np.zeros(n) if sumsq else None
        self._call("CalculateEdgeDerivatives", _ptr(a), _ptr(b), _ptr(d), _ptr(w), n,
                   _ptr(o1), _ptr(o2), _ptr(o3), check=check)
        (self._graph_keep if self._capturing else self._keep).append((o2, o3))
        return (None if o1 is None else o1.reshape(n, self.patternCount)), o2, o3

    def calculateCrossProductDerivative(self, post, pre, crates, cw, lengths, out, check=True):
        """beagleCalculateCrossProductDerivative: adds, over the listed
        branches, the S x S cross-product sums into `out` (float64, S * S,
        row-major; the caller clears it) and returns it."""
        a, b = _i32(post), _i32(pre)
        r, w = _i32(crates), _i32(cw)
        t = _f64(lengths)
        assert out.dtype == np.float64 and out.flags.c_contiguous
        self._call("CalculateCrossProductDerivative", _ptr(a), _ptr(b), _ptr(r), _ptr(w), _ptr(t),
                   len(a), _ptr(out), None, check=check)
        return out

    def supports(self, name):
        """Whether the library exports <prefix><name>."""
        return name in self.blib.fn

    def injectKernelTimeout(self, which):
        """Raise the device flag of a timed-out kernel wait (0: tensor-core
        kernels, 1: bulk-copy derivative); the next result call reports it."""
        self._call("InjectKernelTimeout", which)

    def tunedVariants(self):
        """{kind: variant} the autotuner last ran (beagleB200GetTunedVariants)."""
        o = np.zeros(4, dtype=np.int32)
        self._call("GetTunedVariants", _ptr(o))
        return dict(zip(("post", "pre", "deriv", "fused"), (int(x) for x in o)))

    def updatePartialsWithRootLogLikelihood(self, ops, cumulative, root, cw, sf, check=True):
        """beagleB200UpdatePartialsWithRootLogLikelihood: updatePartials, the
        cumulative scale factors of the list (reset first; -1 for none) and the
        root lnL in one call.  Returns lnL (ASYNCH instances: delivered by
        getLogLikelihood, the return value is then not meaningful)."""
        o = _i32(ops).reshape(-1)
        out = np.zeros(1)
        code = self._call("UpdatePartialsWithRootLogLikelihood", _ptr(o), o.size // 7,
                          cumulative, root, cw, sf, _ptr(out), check=check)
        return (code, float(out[0])) if not check else float(out[0])

    def updatePrePartialsWithDerivatives(self, ops, post, dmat, cw, check=True):
        """Pre-order ops, then the edge derivative of each op's node from
        (post[k], dest of op k, dmat[k]): (sums, sums of squares) in op order
        (beagleB200UpdatePrePartialsWithDerivatives)."""
        o = _i32(ops)
        a, d, w = _i32(post), _i32(dmat), _i32(cw)
        n = len(a)
        o2, o3 = np.zeros(n), np.zeros(n)
        self._call("UpdatePrePartialsWithDerivatives", _ptr(o), n, _ptr(a), _ptr(d), _ptr(w),
                   _ptr(o2), _ptr(o3), check=check)
        (self._graph_keep if self._capturing else self._keep).append((o2, o3))
        return o2, o3

    def calculateEdgeLogLikelihoods(self, parent, child, prob, d1, d2, cw, sf, cum,
                                    check=True):
        arr = [_i32([parent]), _i32([child]), _i32([prob]),
               None if d1 is None else _i32([d1]), None if d2 is None else _i32([d2]),
               _i32([cw]), _i32([sf]), _i32([cum])]
        o = np.zeros(1)
        o1 = np.zeros(1) if d1 is not None else None
        o2 = np.zeros(1) if d2 is not None else None
        code = self._call("CalculateEdgeLogLikelihoods", *[_ptr(x) for x in arr], 1,
                          _ptr(o), _ptr(o1), _ptr(o2), check=check)
        return (code, float(o[0]), None if o1 is None else float(o1[0]),
                None if o2 is None else float(o2[0]))

    def calculateEdgeLogLikelihoodsByPartition(self, parents, children, probs, d1s, d2s, cw,
                                               sf, cum, parts, check=True):
        """Per partition i, the edge lnL of (parents[i], children[i], probs[i])
        over partition parts[i]; d1s / d2s both None (lnL only) or both lists.
        Returns (code, lnL by partition, lnL, d1 by partition or None, d1,
        d2 by partition or None, d2)."""
        p = _i32(parts)
        n = len(p)
        arr = [_i32(parents), _i32(children), _i32(probs),
               None if d1s is None else _i32(d1s), None if d2s is None else _i32(d2s),
               _i32(cw), _i32(sf), _i32(cum), p]
        byp, tot = np.zeros(n), np.zeros(1)
        d1p, d1t = (np.zeros(n), np.zeros(1)) if d1s is not None else (None, None)
        d2p, d2t = (np.zeros(n), np.zeros(1)) if d2s is not None else (None, None)
        code = self._call("CalculateEdgeLogLikelihoodsByPartition", *[_ptr(x) for x in arr], n,
                          1, _ptr(byp), _ptr(tot), _ptr(d1p), _ptr(d1t), _ptr(d2p), _ptr(d2t),
                          check=check)
        return (code, byp, float(tot[0]), d1p, None if d1t is None else float(d1t[0]), d2p,
                None if d2t is None else float(d2t[0]))

    def getLogLikelihood(self, check=True):
        o = np.zeros(1)
        code = self._call("GetLogLikelihood", _ptr(o), check=False)
        self._keep = []
        if check and code < 0 and code != -8:
            raise BeagleError(self.blib.prefix + "GetLogLikelihood", code)
        return float(o[0])

    def getSiteLogLikelihoods(self):
        out = np.zeros(self.patternCount)
        self._call("GetSiteLogLikelihoods", _ptr(out))
        return out

    def cudaStream(self):
        """The instance's cudaStream_t as an int (libbeagle_b200 only)."""
        out = ctypes.c_void_p()
        self._call("GetCudaStream", ctypes.byref(out))
        return out.value or 0

    def getDerivatives(self):
        o1, o2 = np.zeros(1), np.zeros(1)
        self._call("GetDerivatives", _ptr(o1), _ptr(o2))
        self._keep = []
        return float(o1[0]), float(o2[0])

    def getSiteDerivatives(self, second=False):
        o1 = np.zeros(self.patternCount)
        o2 = np.zeros(self.patternCount) if second else None
        self._call("GetSiteDerivatives", _ptr(o1), _ptr(o2))
        return o1, o2


# beagleB200 batch entry points: name -> argument types.
_BATCH_SIGS = {
    "BatchBeginCapture": [_i], "BatchEndCapture": [_i, _p], "BatchLaunchGraph": [_i, _i],
    "CreateBatch": [_p, _i], "FinalizeBatch": [_i],
    "BatchUpdateTransitionMatrices": [_i, _p, _p, _p, _p],
    "BatchUpdatePartials": [_i, _p, _p, _p],
    "BatchUpdatePrePartials": [_i, _p, _p],
    "BatchAccumulateScaleFactors": [_i, _p, _p, _p, _i],
    "BatchSetRootPrePartials": [_i, _p, _p],
    "BatchCalculateRootLogLikelihoods": [_i, _p, _p, _p, _p, _p],
    "BatchCalculateEdgeDerivatives": [_i, _p, _p, _p, _p, _p, _p, _p],
    "BatchWait": [_i],
    "BatchUpdatePrePartialsWithDerivatives": [_i, _p, _p, _p, _p, _p, _p, _p],
    "BatchLaunchGraphWithLengths": [_i, _i, _p, _i],
    "BatchUpdatePartialsWithRootLogLikelihood": [_i, _p, _p, _p, _p, _p, _p, _p],
}


class Batch:
    """A batch of instances of one BeagleLib (``beagleB200*Batch*`` calls):
    per-member arguments are lists indexed by member position."""

    def __init__(self, blib, instances):
        self.blib = blib
        self.members = list(instances)
        lib = blib.lib
        p = blib.prefix
        self._f = {}
        for name, args in _BATCH_SIGS.items():
            f = getattr(lib, p + name)
            f.argtypes = args
            f.restype = _i
            self._f[name] = f
        h = _i32([m.h for m in self.members])
        code = self._f["CreateBatch"](_ptr(h), len(h))
        if code < 0:
            raise BeagleError(p + "CreateBatch", code)
        self.h = code

    def _call(self, name, *args):
        code = self._f[name](self.h, *args)
        if code < 0:
            raise BeagleError(self.blib.prefix + name, code)
        return code

    @staticmethod
    def _ptrs(arrays, dtype):
        """A C array of pointers to contiguous numpy arrays (kept alive by the caller)."""
        keep = [np.ascontiguousarray(a, dtype=dtype) for a in arrays]
        tab = (ctypes.c_void_p * len(keep))(*[a.ctypes.data for a in keep])
        return tab, keep

    def finalize(self):
        if self.h is not None:
            self._f["FinalizeBatch"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.finalize()
        except Exception:
            pass

    def updateTransitionMatrices(self, eigen, prob, lengths):
        pt, k1 = self._ptrs(prob, np.int32)
        lt, k2 = self._ptrs(lengths, np.float64)
        cnt = _i32([len(a) for a in prob])
        return self._call("BatchUpdateTransitionMatrices", _ptr(_i32(eigen)), pt, lt, _ptr(cnt))

    def updatePartials(self, ops, cumulative=None):
        ot, k = self._ptrs([np.asarray(o).reshape(-1) for o in ops], np.int32)
        cnt = _i32([np.asarray(o).size // 7 for o in ops])
        cum = _i32(cumulative) if cumulative is not None else None
        return self._call("BatchUpdatePartials", ot, _ptr(cnt), _ptr(cum))

    def updatePrePartials(self, ops):
        ot, k = self._ptrs([np.asarray(o).reshape(-1) for o in ops], np.int32)
        cnt = _i32([np.asarray(o).size // 7 for o in ops])
        return self._call("BatchUpdatePrePartials", ot, _ptr(cnt))

    def accumulateScaleFactors(self, idx, cumulative, reset=True):
        it, k = self._ptrs(idx, np.int32)
        cnt = _i32([len(a) for a in idx])
        return self._call("BatchAccumulateScaleFactors", it, _ptr(cnt), _ptr(_i32(cumulative)),
                          1 if reset else 0)

    def setRootPrePartials(self, bufs, freqs):
        return self._call("BatchSetRootPrePartials", _ptr(_i32(bufs)), _ptr(_i32(freqs)))

    def wait(self):
        """Deliver deferred results (ASYNCH members) into the arrays returned
        by the result calls."""
        code = self._call("BatchWait")
        self._keep = []
        return code

    # CUDA graphs of batch calls (ASYNCH members)
    def beginCapture(self):
        self._capturing = True
        return self._call("BatchBeginCapture")

    def endCapture(self):
        self._capturing = False
        g = ctypes.c_int(-1)
        self._call("BatchEndCapture", ctypes.byref(g))
        return g.value

    def launchGraph(self, graph):
        return self._call("BatchLaunchGraph", graph)

    def launchGraphWithLengths(self, graph, lengths):
        """New branch lengths for the graph's captured matrix updates (all of
        them, members in batch order), then the graph."""
        t = _f64(lengths)
        return self._call("BatchLaunchGraphWithLengths", graph, _ptr(t), len(t))

    def updatePrePartialsWithDerivatives(self, ops, post, dmat, cw):
        """Per member: the pre-order ops with each op's branch derivative
        (post-order operand post[i][k], derivative matrix dmat[i][k]); returns
        (sums, sums of squares) per member, in op order, filled at wait() for
        ASYNCH members."""
        ot, k1 = self._ptrs([np.asarray(o).reshape(-1) for o in ops], np.int32)
        cnt = _i32([np.asarray(o).size // 7 for o in ops])
        pt, k2 = self._ptrs(post, np.int32)
        dt, k3 = self._ptrs(dmat, np.int32)
        st, k4 = self._ptrs([np.zeros(int(c)) for c in cnt], np.float64)
        qt, k5 = self._ptrs([np.zeros(int(c)) for c in cnt], np.float64)
        self._call("BatchUpdatePrePartialsWithDerivatives", ot, _ptr(cnt), pt, dt, _ptr(_i32(cw)),
                   st, qt)
        self._keep_result(k4, k5)
        return k4, k5

    def _keep_result(self, *arrays):
        """Result arrays stay alive until the wait() that fills them (ASYNCH
        members), and with the batch when a captured call fills them at every
        graph launch."""
        if getattr(self, "_capturing", False):
            self.__dict__.setdefault("_graph_keep", []).append(arrays)
        else:
            self.__dict__.setdefault("_keep", []).append(arrays)

    def calculateRootLogLikelihoods(self, bufs, cw, sf, cum):
        out = np.zeros(len(self.members))
        self._call("BatchCalculateRootLogLikelihoods", _ptr(_i32(bufs)), _ptr(_i32(cw)),
                   _ptr(_i32(sf)), _ptr(_i32(cum)), _ptr(out))
        self._keep_result(out)
        return out

    def updatePartialsWithRootLogLikelihood(self, ops, cumulative, roots, cw, sf):
        """beagleB200BatchUpdatePartialsWithRootLogLikelihood: per member the
        post-order ops, the cumulative scale buffer (reset, then the list's
        scale buffers added; -1 for none) and the root lnL; returns the lnL
        array (filled at wait() for ASYNCH members)."""
        ot, k1 = self._ptrs([np.asarray(o).reshape(-1) for o in ops], np.int32)
        cnt = _i32([np.asarray(o).size // 7 for o in ops])
        out = np.zeros(len(self.members))
        self._call("BatchUpdatePartialsWithRootLogLikelihood", ot, _ptr(cnt),
                   _ptr(_i32(cumulative)), _ptr(_i32(roots)), _ptr(_i32(cw)), _ptr(_i32(sf)),
                   _ptr(out))
        self._keep_result(out)
        return out

    def calculateEdgeDerivatives(self, post, pre, dmat, cw):
        pt, k1 = self._ptrs(post, np.int32)
        qt, k2 = self._ptrs(pre, np.int32)
        dt, k3 = self._ptrs(dmat, np.int32)
        cnt = _i32([len(a) for a in post])
        sums = [np.zeros(len(a)) for a in post]
        sq = [np.zeros(len(a)) for a in post]
        st, k4 = self._ptrs(sums, np.float64)
        qq, k5 = self._ptrs(sq, np.float64)
        self._call("BatchCalculateEdgeDerivatives", pt, qt, dt, _ptr(_i32(cw)), _ptr(cnt), st, qq)
        self._keep_result(k4, k5)
        return k4, k5
