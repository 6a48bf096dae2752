"""Brute-force Lehmann sums and oracle-backed chain runners shared by the GF driver tests
(test infrastructure: imports the oracle)."""
import math

import numpy as np

from ed_lattice_b200.edlat import Spectrum
from oracle import oracle as O


def oracle_chain_fn(m, om):
    """chain_fn for build_gf_electrons from the oracle: apply c/c^+ (sum of two sites for the
    mixed chains), tridiagonalise with the oracle's recurrence, poles and weights."""
    ns = m.ns

    def run(isector, vec, jsector, op, io, jo, ispin, nlanc, ei):
        nup, ndw = m.get_nup(isector), m.get_ndw(isector)
        x = O.apply_cop(ns, nup, ndw, op, io, ispin, vec)
        if jo:
            O.apply_cop(ns, nup, ndw, op, jo, ispin, vec, out=x)
        nj, dj = m.get_nup(jsector), m.get_ndw(jsector)
        st = O.Stored(om, nj, dj)
        a, b, n2, n = st.tridiag(x, min(nlanc, st.dim), 1e-9)
        if n == 0 or n2 == 0.0:
            return Spectrum(np.zeros(0), np.zeros(0), n2)
        p, w = O.poles_weights(a[:n], b[:n], n2, ei, op)
        return Spectrum(p, w, n2)
    return run


def spectra_all_sectors(om, ns):
    out = {}
    for nup in range(ns + 1):
        for ndw in range(ns + 1):
            out[(nup, ndw)] = np.linalg.eigh(O.dense_h(om, nup, ndw))
    return out


def lehmann_g(om, ns, temp, cutoff, finite_temp, pairs, zs, spin=1, spec=None):
    """G_ij(z) for the pairs (1-based sites) summed over the eigenstates kept by the reference's
    rules: every state within the cutoff at finite T, the ground manifold (1e-9) at T=0."""
    spec = spec or spectra_all_sectors(om, ns)
    states = [(w[k], nu, nd, z[:, k]) for (nu, nd), (w, z) in spec.items() for k in range(w.size)]
    egs = min(s[0] for s in states)
    if finite_temp:
        kept = [s for s in states if math.exp(-(s[0] - egs) / temp) > cutoff]
        wts = [math.exp(-(s[0] - egs) / temp) for s in kept]
    else:
        kept = [s for s in states if abs(s[0] - egs) <= 1e-9]
        wts = [1.0] * len(kept)
    zeta = sum(wts)
    g = {pr: np.zeros(len(zs), dtype=np.complex128) for pr in pairs}
    for (en, nu, nd, vec), wt in zip(kept, wts):
        for op in (+1, -1):
            nj = (nu + op, nd) if spin == 1 else (nu, nd + op)
            if not (0 <= nj[0] <= ns and 0 <= nj[1] <= ns):
                continue
            wj, zj = spec[nj]
            amp = {}
            for i in {p for pr in pairs for p in pr}:
                amp[i] = zj.T @ O.apply_cop(ns, nu, nd, op, i, spin, vec)
            de = op * (wj - en)
            for (i, j) in pairs:
                g[(i, j)] += wt / zeta * ((amp[i] * amp[j])[None, :] / (zs[:, None] - de[None, :])).sum(1)
    return g


def exact_channels(om, ns, nup, ndw, vec, ei, apply_op, spec):
    """One same-sector channel with the exact poles E_m - ei and weights |<m|O vec>|^2."""
    w, z = spec[(nup, ndw)]
    amp = z.T @ apply_op(vec)
    return [Spectrum(w - ei, amp * amp, float(amp @ amp))]
