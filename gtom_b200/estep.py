"""RELION E-step consumers (mirror of gtom's d_rlnSquaredDifferences*,
d_rlnConvertWeights*, d_rlnDiffRemap*, d_rlnCreateMinvsigma2s and
d_rlnStoreWeightsAdd, include/Relion.cuh:19-57) on CUDA tensors, over the
C ABI of gtom_b200/csrc/estep.cu.  Arguments keep the reference's order;
complex arrays are complex64 tensors, uint3/uint4 arrays int32/uint32
tensors of 3/4 columns."""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from .relion import _stream


def _p(t):
    if t is None:
        return C.c_void_p(0)
    if not isinstance(t, torch.Tensor) or not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return C.c_void_p(t.data_ptr())


def d_rlnSquaredDifferencesSparse(particleft, minvsigma2, ctf, dimsparticle, precalcshifts, refft, diff2,
                                  combination, ncombinations, groupsize, dofirstitercc=False, stream=None):
    dx, dy, dz = (int(v) for v in dimsparticle)
    _lib.call("gtomrln_squared_differences_sparse", _p(particleft), _p(minvsigma2), _p(ctf), dx, dy, dz,
              _p(precalcshifts), _p(refft), _p(diff2), _p(combination), int(ncombinations), int(groupsize),
              int(bool(dofirstitercc)), _stream(stream))


def d_rlnSquaredDifferences(particleft, minvsigma2, ctf, dimsparticle, nparticles, precalcshifts, nshifts, refft,
                            nrefs, tile, diff2, dofirstitercc=False, stream=None):
    dx, dy, dz = (int(v) for v in dimsparticle)
    _lib.call("gtomrln_squared_differences", _p(particleft), _p(minvsigma2), _p(ctf), dx, dy, dz, int(nparticles),
              _p(precalcshifts), int(nshifts), _p(refft), int(nrefs), int(tile), _p(diff2),
              int(bool(dofirstitercc)), _stream(stream))


def d_rlnConvertWeightsDense(weights, nparticles, nclasses, nrot, ntrans, pdfrot, pdftrans, mindiff2, stream=None):
    _lib.call("gtomrln_convert_weights_dense", _p(weights), int(nparticles), int(nclasses), int(nrot), int(ntrans),
              _p(pdfrot), _p(pdftrans), _p(mindiff2), _stream(stream))


def d_rlnConvertWeightsSparse(weightsdense, weightssparse, combinations, nsparse, nrot, ntrans, pdfrot, pdftrans,
                              mindiff2, stream=None):
    _lib.call("gtomrln_convert_weights_sparse", _p(weightsdense), _p(weightssparse), _p(combinations),
              int(nsparse), int(nrot), int(ntrans), _p(pdfrot), _p(pdftrans), _p(mindiff2), _stream(stream))


def d_rlnConvertWeightsSort(inp, n, stream=None):
    _lib.call("gtomrln_convert_weights_sort", _p(inp), int(n), _stream(stream))


def d_rlnConvertWeightsCompact(inp, out, n, stream=None) -> int:
    """Returns the number of positive values copied (the reference's in/out n)."""
    c = C.c_uint(int(n))
    _lib.call("gtomrln_convert_weights_compact", _p(inp), _p(out), C.byref(c), _stream(stream))
    return c.value


def d_rlnDiffRemapDense(inp, out, orientationindices, norientations, iclass, nparticles, nclasses, nrot, ntrans,
                        ntranspadded, xi2imgs, sqrtxi2, docc=False, stream=None):
    _lib.call("gtomrln_diff_remap_dense", _p(inp), _p(out), _p(orientationindices), int(norientations),
              int(iclass), int(nparticles), int(nclasses), int(nrot), int(ntrans), int(ntranspadded), _p(xi2imgs),
              _p(sqrtxi2), int(bool(docc)), _stream(stream))


def d_rlnDiffRemapSparse(inp, out, mindiff2, combinations, hiddenover, elements, tileelements, weightsperpart,
                         nparticles, xi2imgs, sqrtxi2, docc=False, stream=None):
    _lib.call("gtomrln_diff_remap_sparse", _p(inp), _p(out), _p(mindiff2), _p(combinations), _p(hiddenover),
              int(elements), int(tileelements), int(weightsperpart), int(nparticles), _p(xi2imgs), _p(sqrtxi2),
              int(bool(docc)), _stream(stream))


def d_rlnCreateMinvsigma2s(out, mresol, elements, sigma2noise, sigma2fudge, stream=None):
    _lib.call("gtomrln_create_minvsigma2s", _p(out), _p(mresol), int(elements), _p(sigma2noise),
              C.c_float(float(sigma2fudge)), _stream(stream))


def d_rlnStoreWeightsAdd(inp, ctf, ref, minvsigma2, mresol, elements, ntrans, weights, sigweight, sumweight,
                         output, outputweights, sigma2noise, normcorrection, priorclass, correctionxa,
                         correctionaa, doscale, stream=None):
    _lib.call("gtomrln_store_weights_add", _p(inp), _p(ctf), _p(ref), _p(minvsigma2), _p(mresol), int(elements),
              int(ntrans), _p(weights), C.c_float(float(sigweight)), C.c_float(float(sumweight)), _p(output),
              _p(outputweights), _p(sigma2noise), _p(normcorrection), _p(priorclass), _p(correctionxa),
              _p(correctionaa), int(bool(doscale)), _stream(stream))
