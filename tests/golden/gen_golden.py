"""Generate the golden fixtures of tests/golden/ from the reference's own CPU
libraries (oracle/_ref, compiled from the reference sources by oracle/Makefile).

Each fixture stores the inputs (the OTF network as flat arrays, basis
parameters, seeded vectors, angles) and the reference outputs of
hvec_gather_contract_otf_f64, get_diags_elements_f64, expm/grad/backgrad/
batch_grad_contract_otf_f64, tvec/backtran/batch_expm/batch_tran_contract_otf_f64
and a few libdiag helpers.  Run:

    python tests/golden/gen_golden.py

Small sizes only (dim <= 4900) so the fixtures stay a few hundred KB.
`python tests/golden/gen_golden.py --c64` writes the complex-interface fixture
(c64_h6_3a2b.npz) from the _c64 entry points.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from binsim_b200 import network as nw  # noqa: E402
from oracle.oracle import RefLibs, build_ref  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

CASES = [
    # name, norb, na, nb, orbsym, total_sym, num_irreps, seed
    ("h6_3a3b", 6, 3, 3, None, 0, 16, 11),
    ("h8_4a3b_sym", 8, 4, 3, [0, 1, 0, 1, 2, 3, 2, 3], 1, 4, 12),
    ("h8_4a4b", 8, 4, 4, None, 0, 16, 13),
]


def net_arrays(prefix, net):
    return {f"{prefix}_{k}": np.asarray(getattr(net, k)) for k in
            ("orbsym", "axs", "bxs", "ranks", "num_zas", "num_zbs", "flat_zas", "flat_zbs", "flat_wa", "flat_wb")} | \
        {f"{prefix}_norb": np.asarray(net.norb)}


def main():
    if not build_ref():
        raise SystemExit("reference libraries unavailable (need the reference sources)")
    ref = RefLibs()
    for name, norb, na, nb, orbsym, tsym, nirr, seed in CASES:
        ham = nw.hamiltonian_network(norb, seed=seed)
        pool = nw.ucc_pool(norb).network
        osym = np.zeros(norb, np.int64) if orbsym is None else np.asarray(orbsym, np.int64)
        ham.orbsym = osym
        pool.orbsym = osym
        rb, dim = ref.basis(norb, na, nb, orbsym=osym, total_sym=tsym, num_irreps=nirr)
        rh, rp = ref.network(ham), ref.network(pool)
        rng = np.random.default_rng(seed)
        x = rng.normal(size=dim); x /= np.linalg.norm(x)
        y = rng.normal(size=dim); y /= np.linalg.norm(y)
        sigma = ref.hvec(rb, rh, x, dim)
        diag = ref.diag_elems(rb, rh, dim)
        ops = rng.choice(pool.ngs, size=min(12 if dim <= 1000 else 4, pool.ngs), replace=False)
        thetas = rng.normal(0, 0.7, size=len(ops))
        expm = np.stack([ref.expm(rb, rp, int(i), t, x) for i, t in zip(ops, thetas)])
        grad = np.array([ref.grad(rb, rp, int(i), t, x, y) for i, t in zip(ops, thetas)])
        bg = [ref.backgrad(rb, rp, int(i), t, x, y) for i, t in zip(ops, thetas)]
        bth = rng.normal(0, 0.3, size=pool.ngs)
        batch = ref.batchgrad(rb, rp, bth, x, sigma, pool.ngs)
        hf = ref.det_index(rb, (1 << na) - 1, (1 << nb) - 1, dim)
        # tvec / backtran / batch_expm / batch_tran (drawn after the arrays above,
        # so those stay as they were): pool generators and the diagonal group 0
        # of the Hamiltonian
        top = ops[:4]
        tvec = np.stack([ref.tvec(rb, rp, int(i), x, dim) for i in top])
        tvec_ham0 = ref.tvec(rb, rh, 0, x, dim)
        bt = [ref.backtran(rb, rp, int(i), t, x, y, dim) for i, t in zip(top, thetas[:4])]
        bt_ham0 = ref.backtran(rb, rh, 0, 0.4, x, y, dim)
        bem = rng.normal(size=(dim, 3))
        bexp = ref.batchexpm(rb, rp, int(ops[0]), float(thetas[0]), bem, 2)
        trans_pool = ref.batchtran(rb, rp, x, y, pool.ngs)
        trans_ham = ref.batchtran(rb, rh, x, y, ham.ngs)
        np.savez_compressed(
            os.path.join(OUT, f"{name}.npz"),
            norb=norb, na=na, nb=nb, orbsym=osym, total_sym=tsym, num_irreps=nirr, dim=dim, hf=hf,
            x=x, y=y, sigma=sigma, diag=diag, ops=ops, thetas=thetas, expm=expm, grad=grad,
            backgrad=np.array([b[0] for b in bg]), backgrad_l=np.stack([b[1] for b in bg]),
            backgrad_r=np.stack([b[2] for b in bg]), batch_thetas=bth, batchgrad=batch,
            tvec=tvec, tvec_ham0=tvec_ham0, backtran_l=np.stack([b[0] for b in bt]),
            backtran_r=np.stack([b[1] for b in bt]), backtran_b=np.stack([b[2] for b in bt]),
            backtran_ham0=np.stack(bt_ham0), batchexpm_in=bem, batchexpm=bexp, trans_pool=trans_pool,
            trans_ham=trans_ham,
            **net_arrays("ham", ham), **net_arrays("pool", pool))
        print(name, "dim", dim, "ham groups", ham.ngs, "pool groups", pool.ngs)


def complex_weights(net, seed):
    """Each real weight times a seeded modulus in [0.5, 1.5) and phase."""
    rng = np.random.default_rng(seed)
    n_a, n_b = len(net.flat_wa), len(net.flat_wb)
    wa = np.asarray(net.flat_wa) * rng.uniform(0.5, 1.5, n_a) * np.exp(1j * rng.uniform(0, 6.3, n_a))
    wb = np.asarray(net.flat_wb) * rng.uniform(0.5, 1.5, n_b) * np.exp(1j * rng.uniform(0, 6.3, n_b))
    return wa, wb


def main_c64():
    """c64_h6_3a2b.npz: the reference's complex interface (Tv = complex<double>) on a
    6-orbital 3a+2b space with symmetry blocks: complex-weight Hamiltonian and pool."""
    ref = RefLibs()
    norb, na, nb, tsym, nirr = 6, 3, 2, 1, 4
    osym = np.array([0, 1, 0, 1, 2, 3], np.int64)
    ham = nw.hamiltonian_network(norb, seed=31)
    pool = nw.ucc_pool(norb).network
    ham.orbsym = osym
    pool.orbsym = osym
    hwa, hwb = complex_weights(ham, 1)
    pwa, pwb = complex_weights(pool, 2)
    rb, dim = ref.basis(norb, na, nb, orbsym=osym, total_sym=tsym, num_irreps=nirr)
    rh, rp = ref.network_c64(ham, hwa, hwb), ref.network_c64(pool, pwa, pwb)
    rng = np.random.default_rng(5)
    x = rng.normal(size=dim) + 1j * rng.normal(size=dim)
    y = rng.normal(size=dim) + 1j * rng.normal(size=dim)
    ops = rng.choice(pool.ngs, size=6, replace=False)
    thetas = rng.normal(0, 0.7, size=6)
    bg = [ref.backgrad_c64(rb, rp, int(i), t, x, y) for i, t in zip(ops, thetas)]
    bt = [ref.backtran_c64(rb, rp, int(i), t, x, y, dim) for i, t in zip(ops, thetas)]
    M = rng.normal(size=(dim, 3)) + 1j * rng.normal(size=(dim, 3))
    bth = rng.normal(0, 0.3, size=pool.ngs)
    np.savez_compressed(
        os.path.join(OUT, "c64_h6_3a2b.npz"),
        norb=norb, na=na, nb=nb, orbsym=osym, total_sym=tsym, num_irreps=nirr, dim=dim, x=x, y=y,
        ham_wa=hwa, ham_wb=hwb, pool_wa=pwa, pool_wb=pwb,
        sigma=ref.hvec_c64(rb, rh, x, dim), diag=ref.diag_c64(rb, rh, dim),
        expm_ham0=ref.expm_c64(rb, rh, 0, 0.6, x), grad_ham0=ref.grad_c64(rb, rh, 0, 0.6, x, y),
        ops=ops, thetas=thetas,
        expm=np.stack([ref.expm_c64(rb, rp, int(i), t, x) for i, t in zip(ops, thetas)]),
        grad=np.array([ref.grad_c64(rb, rp, int(i), t, x, y) for i, t in zip(ops, thetas)]),
        backgrad=np.array([b[0] for b in bg]), backgrad_l=np.stack([b[1] for b in bg]),
        backgrad_r=np.stack([b[2] for b in bg]),
        tvec=np.stack([ref.tvec_c64(rb, rp, int(i), x, dim) for i in ops]),
        tvec_ham0=ref.tvec_c64(rb, rh, 0, x, dim),
        backtran_l=np.stack([b[0] for b in bt]), backtran_r=np.stack([b[1] for b in bt]),
        backtran_b=np.stack([b[2] for b in bt]),
        batchexpm_in=M, batchexpm=ref.batchexpm_c64(rb, rp, int(ops[0]), float(thetas[0]), M, 2),
        batch_thetas=bth, batchgrad=ref.batchgrad_c64(rb, rp, bth, x, y, pool.ngs),
        trans_pool=ref.batchtran_c64(rb, rp, x, y, pool.ngs), trans_ham=ref.batchtran_c64(rb, rh, x, y, ham.ngs),
        **net_arrays("ham", ham), **net_arrays("pool", pool))
    print("c64_h6_3a2b dim", dim, "ham groups", ham.ngs, "pool groups", pool.ngs)


if __name__ == "__main__":
    if "--c64" in sys.argv:
        main_c64()
    else:
        main()
