"""Generate the committed golden fixtures under tests/golden/ from the CPU oracle.

The reference (Fortran + SciFortran) cannot be built or run on this machine and ships no
fixtures, so these vectors come from oracle/edlat_oracle.cpp, whose own correctness is
pinned by known answers in tests/test_oracle_known_answers.py. They freeze the oracle's
outputs (regression) and give the GPU tests fixed expected values that do not depend on
rebuilding the oracle on the GPU host.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def ring(L, t=1.0):
    H = np.zeros((L, L))
    for i in range(L):
        j = (i + 1) % L
        H[i, j] = H[j, i] = -t
    return H


def square(lx, ly, t=1.0):
    ns = lx * ly
    H = np.zeros((ns, ns))
    for y in range(ly):
        for x in range(lx):
            i = x + lx * y
            for dx, dy in ((1, 0), (0, 1)):
                j = (x + dx) % lx + lx * ((y + dy) % ly)
                if i != j:
                    H[i, j] = H[j, i] = -t
    return H


def ring8():
    """L=8 periodic ring, t=1, U=4, mu=U/2 (HFMODE=F, XMU=2), sector (4,4), FP64,
    seeded uniform[-1,1) start vector (seed 2024), 100 tridiagonal steps."""
    m = O.Model(ring(8), uloc=4.0, xmu=2.0, hfmode=False)
    st = O.Stored(m, 4, 4)
    v0 = O.random_vector(2024, st.dim)
    a, b, n2, n = st.tridiag(v0, 100)
    e0, vec, ga, gb = st.ground_state(v0, maxit=300, tol=1e-15)
    obs = O.observables(8, 4, 4, vec)
    hv = st.matvec_d(v0)
    hvd = O.direct_matvec_d(m, 4, 4, v0)
    np.savez_compressed(os.path.join(HERE, "ring8_U4_sector44.npz"), v0=v0, hv_stored=hv, hv_direct=hvd, alanc=a,
                        blanc=b, norm2=n2, e0=e0, dens=obs["dens"], docc=obs["docc"],
                        map_up=O.build_map(8, 4))


def disorder3x4():
    """3x4 periodic square, t=1, U=4, Anderson eps_i ~ uniform[-1,1) quantised to 2^-16
    (seed 7), XMU=2 HFMODE=F; sector (3,2): maps, hop tables, H x v, E0 and a GF chain."""
    rng = np.random.default_rng(7)
    eps = np.round(rng.uniform(-1, 1, 12) * 65536) / 65536
    H = square(3, 4)
    H[np.diag_indices(12)] = eps
    m = O.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    st = O.Stored(m, 3, 2)
    v0 = O.random_vector(99, st.dim)
    hv = st.matvec_d(v0)
    rp_up, c_up, v_up = O.hop_csr(m, 1, 3)
    rp_dw, c_dw, v_dw = O.hop_csr(m, 2, 2)
    e0, vec, _, _ = st.ground_state(v0, maxit=400, tol=1e-15)
    # c^+_{5,up}|GS> into (4,2), 60 steps
    x = O.apply_cop(12, 3, 2, +1, 5, 1, vec)
    stJ = O.Stored(m, 4, 2)
    a, b, n2, n = stJ.tridiag(x, 60, 1e-9)
    p, w = O.poles_weights(a[:n], b[:n], n2, e0, +1)
    np.savez_compressed(os.path.join(HERE, "disorder3x4.npz"), eps=eps, v0=v0, hv=hv, rp_up=rp_up, c_up=c_up,
                        v_up=v_up, rp_dw=rp_dw, c_dw=c_dw, v_dw=v_dw, e0=e0, gs_vec=vec, gf_poles=p, gf_weights=w,
                        gf_norm2=n2)


def thermal3x4():
    """The disorder3x4 lattice over all 169 (Nup,Ndw) sectors: the lowest 4 levels of each
    sector, then the finite-temperature state list at beta=20 (T=0.05, cutoff 1e-9) with Z and
    the thermal n_i, n_i,up, n_i,dw, d_i, m_i. Sectors with D <= 4000 are diagonalised densely
    (scipy.linalg.eigh on the oracle's dense matrix); larger ones with ARPACK (scipy's eigsh,
    the library behind the reference's sp_eigh) over the oracle's stored H x v."""
    import math

    import scipy.linalg as sla
    import scipy.sparse.linalg as spla

    rng = np.random.default_rng(7)
    eps = np.round(rng.uniform(-1, 1, 12) * 65536) / 65536
    H = square(3, 4)
    H[np.diag_indices(12)] = eps
    m = O.Model(H, uloc=4.0, xmu=2.0, hfmode=False)
    ns, k, temp, cutoff = 12, 4, 0.05, 1e-9
    energies = np.full(((ns + 1) ** 2, k), np.nan)
    dims = np.zeros((ns + 1) ** 2, dtype=np.int64)
    states = []
    for isector in range(1, (ns + 1) ** 2 + 1):
        nup, ndw = O.lib().orc_get_nup(ns, isector), O.lib().orc_get_ndw(ns, isector)
        D = O.binomial(ns, nup) * O.binomial(ns, ndw)
        dims[isector - 1] = D
        kk = min(k, D)
        if D <= 4000:
            w, z = sla.eigh(O.dense_h(m, nup, ndw), subset_by_index=[0, kk - 1])
        else:
            st = O.Stored(m, nup, ndw)
            op = spla.LinearOperator((D, D), matvec=lambda v, st=st: st.matvec_d(np.ascontiguousarray(v)),
                                     dtype=np.float64)
            w, z = spla.eigsh(op, k=kk, which="SA", tol=1e-13, ncv=40, v0=O.random_vector(5, D), maxiter=5000)
            order = np.argsort(w)
            w, z = w[order], z[:, order]
        energies[isector - 1, :kk] = w
        states += [(w[i], isector, nup, ndw, z[:, i]) for i in range(kk)]
        print(f"sector ({nup},{ndw}) D={D} E={w}", flush=True)
    states.sort(key=lambda s: s[0])
    egs = states[0][0]
    kept = [s for s in states if math.exp(-(s[0] - egs) / temp) > cutoff]
    zeta = sum(math.exp(-(s[0] - egs) / temp) for s in kept)
    acc = {q: np.zeros(ns) for q in ("dens", "dens_up", "dens_dw", "docc", "magz")}
    for e, _, nup, ndw, v in kept:
        o = O.observables(ns, nup, ndw, v, math.exp(-(e - egs) / temp) / zeta)
        for q in acc:
            acc[q] += o[q]
    np.savez_compressed(os.path.join(HERE, "thermal3x4.npz"), eps=eps, dims=dims, energies=energies, egs=egs,
                        zeta=zeta, nkept=len(kept), kept_sectors=np.array([s[1] for s in kept]),
                        kept_energies=np.array([s[0] for s in kept]), **acc)


if __name__ == "__main__":
    which = sys.argv[1:] or ["ring8", "disorder3x4", "thermal3x4"]
    for name in which:
        globals()[name]()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")
