"""Test infrastructure: float64 numpy restatements of the RELION E-step
consumers (gtom's src/Relion/ConvertWeights.cu, DiffRemap.cu, Misc.cu,
StoreWeights.cu) and of the squared differences, which gtom declares but
does not define (include/Relion.cuh:46-48; the computation follows the CPU
loop of GTOMTest/RelionSquaredDiff.cpp:55-69).  Only tests may import it."""
from __future__ import annotations

import numpy as np


def squared_differences_sparse(particle, minvsigma2, ctf, shifts, refs, combos, group, cc=False):
    """particle: (nparticles, e) complex; shifts (nshifts, e); refs (nrefs, e);
    combos (k, 3) = (first shift, particle, first ref).  Returns (k*g*g,)."""
    particle = np.asarray(particle, np.complex128)
    e = particle.shape[-1]
    w = np.ones(e) if minvsigma2 is None else np.asarray(minvsigma2, np.float64)
    out = []
    for s0, p, r0 in np.asarray(combos).reshape(-1, 3):
        c = np.ones(e) if ctf is None else np.asarray(ctf, np.float64).reshape(-1, e)[p]
        for r in range(group):
            a = c * np.asarray(refs[r0 + r], np.complex128)
            for s in range(group):
                b = particle[p] * np.asarray(shifts[s0 + s], np.complex128)
                if cc:
                    out.append(-np.sum((a * np.conj(b)).real) / np.sqrt(np.sum(np.abs(a) ** 2)))
                else:
                    out.append(0.5 * np.sum(w * np.abs(a - b) ** 2))
    return np.array(out)


def squared_differences_dense(particle, minvsigma2, ctf, shifts, refs, cc=False):
    """(nparticles, nrefs, nshifts) of the same quantity."""
    particle = np.asarray(particle, np.complex128)
    npart = particle.shape[0]
    out = np.zeros((npart, len(refs), len(shifts)))
    for p in range(npart):
        for r in range(len(refs)):
            for s in range(len(shifts)):
                out[p, r, s] = squared_differences_sparse(particle, minvsigma2, ctf, shifts, refs, [(s, p, r)], 1,
                                                          cc)[0]
    return out


def convert_weights_dense(weights, nparticles, nclasses, nrot, ntrans, pdfrot, pdftrans, mindiff2):
    w = np.asarray(weights, np.float64).reshape(nparticles, nclasses, nrot, ntrans)
    pr = np.asarray(pdfrot, np.float64).reshape(nclasses, nrot)
    pt = np.asarray(pdftrans, np.float64).reshape(nparticles, nclasses, ntrans)
    md = np.asarray(mindiff2, np.float64).reshape(nparticles)
    return (pr[None, :, :, None] * pt[:, :, None, :] * np.exp(-(w - md[:, None, None, None]))).ravel()


def convert_weights_sparse(dense, combos, nrot, ntrans, pdfrot, pdftrans, mindiff2):
    d = np.asarray(dense, np.float64).copy()
    c = np.asarray(combos).reshape(-1, 4)
    pr, pt = np.asarray(pdfrot, np.float64), np.asarray(pdftrans, np.float64)
    sparse = pr[c[:, 0] * nrot + c[:, 1]] * pt[c[:, 0] * ntrans + c[:, 2]] * np.exp(-(d[c[:, 3]] - float(mindiff2)))
    d[c[:, 3]] = sparse
    return d, sparse


def diff_remap_dense(inp, orient, iclass, nparticles, nclasses, nrot, ntrans, ntranspadded, xi2, sqrtxi2, cc,
                     out):
    inp = np.asarray(inp, np.float64).reshape(-1, nparticles, ntranspadded)
    out = np.array(out, np.float64).reshape(nparticles, nclasses, nrot, ntrans)
    o = np.asarray(orient).reshape(-1, 3)
    for irot in range(len(o)):
        v = inp[irot, :, :ntrans]
        v = v * np.asarray(sqrtxi2)[:, None] if cc else v + np.asarray(xi2)[:, None]
        out[:, iclass, o[irot, 1], :] = v
    return out.ravel()


def diff_remap_sparse(inp, combos, hiddenover, tileelements, weightsperpart, xi2, sqrtxi2, cc, out, mindiff2):
    inp = np.asarray(inp, np.float64)
    out = np.array(out, np.float64)
    md = np.array(mindiff2, np.float64)
    part = np.asarray(combos).reshape(-1, 3)[np.arange(len(inp)) // tileelements, 1]
    v = inp * np.asarray(sqrtxi2)[part] if cc else inp + np.asarray(xi2)[part]
    out[weightsperpart * part + np.asarray(hiddenover)] = v
    np.minimum.at(md, part, v)
    return out, md


def create_minvsigma2s(mresol, sigma2noise, fudge):
    r = np.asarray(mresol)
    s = np.asarray(sigma2noise, np.float64)
    return np.where(r > 0, 1.0 / (fudge * s[np.maximum(r, 0)]), 0.0)


def store_weights_add(inp, ctf, ref, minvsigma2, mresol, weights, sigweight, sumweight, output, outweights,
                      sigma2noise, normcorr, priorclass, corrxa, corraa, doscale):
    inp = np.asarray(inp, np.complex128)
    output = np.array(output, np.complex128)
    outweights = np.array(outweights, np.float64)
    s2, nc = np.array(sigma2noise, np.float64), np.array(normcorr, np.float64)
    xa, aa = np.array(corrxa, np.float64), np.array(corraa, np.float64)
    c, w2, r = np.asarray(ctf, np.float64), np.asarray(minvsigma2, np.float64), np.asarray(ref, np.complex128)
    res = np.asarray(mresol)
    pc = np.asarray(priorclass, np.float64)
    for t, wt in enumerate(np.asarray(weights, np.float64)):
        if wt >= sigweight:
            wt = wt * (1.0 / sumweight)
            wx = wt * c * w2
            output[t] += inp[t] * wx
            outweights[t] += wx * c
            ok = res > -1
            d = np.abs(r - inp[t]) ** 2 * wt
            np.add.at(s2, res[ok], d[ok])
            nc[0] += d[ok].sum()
            if doscale:
                ok2 = ok & (pc[np.maximum(res, 0)] > 3)
                np.add.at(xa, res[ok2], (wt * (r * np.conj(inp[t])).real)[ok2])
                np.add.at(aa, res[ok2], (wt * np.abs(r) ** 2)[ok2])
        else:
            output[t] = 0
            outweights[t] = 0
    return output, outweights, s2, nc, xa, aa
