"""Pool-gradient plan (bsim_poolplan_classify, host code): every pool group recognised as
coef * (t - t^dagger) for one spin-orbital excitation, and the pool gradient at theta = 0
rebuilt from five transition-density tables (tests/_tdm_ref.py) against the reference's
batch_tran outputs (golden) and the oracle's batch_grad."""
import numpy as np
import pytest

from binsim_b200 import cuotf, network as nw
from conftest import load_golden

import _tdm_ref as tdm


def _normal_form(cre, ann):
    """(kind, idx, sign) of t = a+_{cre..} a_{ann..} in alpha-first order (spin orbital
    2p + s), written independently of the library."""
    ops = [(m, True) for m in cre] + [(m, False) for m in ann]
    inv = sum(1 for i in range(len(ops)) for j in range(i + 1, len(ops)) if ops[i][0] % 2 and not ops[j][0] % 2)
    oa = [m // 2 for m, _ in ops if m % 2 == 0]
    ob = [m // 2 for m, _ in ops if m % 2 == 1]
    kind = {(2, 0): 1, (0, 2): 2, (2, 2): 3, (4, 0): 4, (0, 4): 5}[(len(oa), len(ob))]
    idx = (oa + ob + [0, 0, 0, 0])[:4]
    return kind, idx, (-1.0) ** inv


_DAG = {1: (1, 0, 2, 3), 2: (1, 0, 2, 3), 3: (1, 0, 3, 2), 4: (3, 2, 1, 0), 5: (3, 2, 1, 0)}


def _canon(kind, idx, coef):
    """Same-spin doubles are antisymmetric in (p, q) and in (r, s): order each pair
    descending, with the sign."""
    idx = [int(v) for v in idx]
    if kind in (4, 5):
        if idx[0] < idx[1]:
            idx[0], idx[1], coef = idx[1], idx[0], -coef
        if idx[2] < idx[3]:
            idx[2], idx[3], coef = idx[3], idx[2], -coef
    return idx, coef


def _same_generator(kind, idx, coef, want):
    """Plan entry equals (kind, idx, sign) up to orientation: coef (X[dag] - X[idx]) is
    unchanged when idx and its dagger swap and coef changes sign."""
    k, ix, s = want
    if kind != k:
        return False
    got, c = _canon(k, idx, coef)
    fwd, sf = _canon(k, ix, s)
    dag, sd = _canon(k, [ix[j] for j in _DAG[k]], s)
    return (got == fwd and abs(c - sf) < 1e-12) or (got == dag and abs(c + sd) < 1e-12)


@pytest.mark.parametrize("norb", [4, 7])
def test_plan_recovers_every_pool_excitation(norb):
    pool = nw.ucc_pool(norb)
    kind, idx, coef = cuotf.pool_plan(pool.network)
    assert len(pool.excitations) == pool.network.ngs
    for g, (cre, ann) in enumerate(pool.excitations):
        assert _same_generator(kind[g], idx[g], coef[g], _normal_form(cre, ann)), (g, cre, ann)


@pytest.mark.parametrize("case", ["h6_3a3b", "h8_4a4b"])
def test_density_gradient_matches_reference_batch_tran(case):
    """Golden trans_pool = the reference library's batch_tran_contract_otf(x, y), which is
    the theta = 0 pool gradient for groups without a diagonal part."""
    z, _, pool = load_golden(case)
    from oracle.oracle import Oracle
    B = Oracle().basis(int(z["norb"]), int(z["na"]), int(z["nb"]))
    assert B.num_blocks == 1 and B.dim == int(z["dim"])
    kind, idx, coef = cuotf.pool_plan(pool)
    assert np.all(kind > 0)
    tb = tdm.tables(B.strings(0, 0), B.strings(0, 1), z["x"], z["y"], pool.norb)
    g = tdm.grads_from_plan(tb, kind, idx, coef)
    ref = z["trans_pool"]
    assert np.abs(g - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("norb,na,nb", [(5, 2, 3), (6, 3, 2)])
def test_density_gradient_matches_oracle_batchgrad(oracle, norb, na, nb):
    pool = nw.ucc_pool(norb)
    net = pool.network
    rng = np.random.default_rng(norb + na)
    scale = rng.uniform(-2.0, 2.0, net.ngs)            # group g becomes scale_g * (t - t^dagger)
    wa = net.flat_wa.copy()
    off = 0
    for g in range(net.ngs):
        n = int(net.num_zas[g] * net.ranks[g])
        wa[off:off + n] *= scale[g]
        off += n
    net2 = nw.OTFNetwork(**{**net.__dict__, "flat_wa": wa})
    kind, idx, coef = cuotf.pool_plan(net2)
    assert np.all(kind > 0)
    for g, (cre, ann) in enumerate(pool.excitations):
        k, ix, sg = _normal_form(cre, ann)
        assert _same_generator(kind[g], idx[g], coef[g] / scale[g], (k, ix, sg)), g
    B = oracle.basis(norb, na, nb)
    l, r = rng.normal(size=B.dim), rng.normal(size=B.dim)
    ref = oracle.batchgrad(B, oracle.network(net2), np.zeros(net2.ngs), l, r)
    g = tdm.grads_from_plan(tdm.tables(B.strings(0, 0), B.strings(0, 1), l, r, norb), kind, idx, coef)
    assert np.abs(g - ref).max() <= 1e-13 * np.abs(ref).max()


def test_hamiltonian_groups_are_not_excitations():
    """Hermitian groups (t + t^dagger, many-term sums) match no generator: general or zero."""
    kind, _, _ = cuotf.pool_plan(nw.hamiltonian_network(6, seed=2))
    assert set(np.unique(kind)) <= {-1, 0} and (kind == 0).sum() == 1


def test_plan_beyond_32_orbitals():
    """Masks past spin orbital 63 (the two-word interleaved form): 40 orbitals."""
    norb = 40
    keys = [((2 * 39, 2 * 3 + 1), (2 * 20 + 1, 2 * 0)), ((2 * 38 + 1,), (2 * 31 + 1,)),
            ((2 * 35, 2 * 33), (2 * 34, 2 * 1)), ((2 * 36 + 1, 2 * 2 + 1), (2 * 2 + 1, 2 * 30 + 1))]
    ax, az, bx, bz, cc, sizes = [], [], [], [], [], []
    by_shape = {}
    for i, (cr, an) in enumerate(keys):
        by_shape.setdefault((len(cr), len(an)), []).append(i)
    terms = [None] * len(keys)
    for _, ids in by_shape.items():
        for i, t in zip(ids, nw._components_batch([keys[i] for i in ids], norb)):
            terms[i] = t
    for t in terms:
        ax.append(t[0]); az.append(t[1]); bx.append(t[2]); bz.append(t[3]); cc.append(t[4]); sizes.append(len(t[4]))
    net = nw._compress_each(*[np.concatenate(v) for v in (ax, az, bx, bz, cc)], sizes, norb)
    kind, idx, coef = cuotf.pool_plan(net)
    for g, (cre, ann) in enumerate(keys):
        assert _same_generator(kind[g], idx[g], coef[g], _normal_form(cre, ann)), g


def test_plan_argument_checks():
    L = cuotf.lib()
    z = np.zeros(4, np.int64)
    assert L.bsim_poolplan_classify(4, 0, *([None] * 12)) == 0
    assert L.bsim_poolplan_classify(4, 1, *([None] * 12)) == -1
    assert L.bsim_poolplan_classify(65, 1, *([z.ctypes.data] * 12)) == -2
    assert L.bsim_poolplan_classify(4, -1, *([z.ctypes.data] * 12)) == -2


@pytest.mark.parametrize("norb,ne,holes", [(6, 3, 1), (6, 3, 2), (7, 2, 2), (9, 4, 1), (40, 3, 2)])
def test_library_hole_tables(norb, ne, holes):
    """bsim_pooldensity_hole_table against the CPU statement's hole tables: same hole
    strings (increasing), same created-string indices and signs, -1 where a created
    orbital is occupied."""
    import itertools
    strs = np.array(sorted(sum(1 << o for o in c) for c in itertools.combinations(range(norb), ne)), np.uint64)
    nh, tab = cuotf.hole_table(strs, norb, holes)
    if norb > 12:   # the itertools tables of the CPU statement are too large here: spot checks
        where = {int(s): i for i, s in enumerate(strs)}
        rng = np.random.default_rng(0)
        for h in rng.choice(nh, 20, replace=False):
            for j in rng.choice(tab.shape[1], 30, replace=False):
                e = int(tab[h, j])
                x = int((np.sqrt(8 * j + 1) + 1) // 2)
                while x * (x - 1) // 2 > j:
                    x -= 1
                y = j - x * (x - 1) // 2
                s = int(strs[e >> 1]) if e >= 0 else None
                if e >= 0:
                    hs = s ^ (1 << x) ^ (1 << y)
                    sg, s2 = tdm._create(hs, [x, y])
                    assert s2 == s and (sg < 0) == bool(e & 1) and where[s] == e >> 1
        return
    idx, sgn = tdm.hole_table(strs, holes, norb)
    assert nh == idx.shape[0]
    if holes == 1:
        want = np.where(sgn != 0, (idx << 1) | (sgn < 0), -1)
    else:
        pairs = [(x, y) for x in range(norb) for y in range(x)]
        cols = [x * norb + y for x, y in pairs]
        want = np.where(sgn[:, cols] != 0, (idx[:, cols] << 1) | (sgn[:, cols] < 0), -1)
        order = np.argsort([x * (x - 1) // 2 + y for x, y in pairs])
        want = want[:, order]
    assert np.array_equal(tab, want)


@pytest.mark.parametrize("norb,na,nb", [(5, 2, 3), (6, 3, 3), (6, 1, 2)])
def test_device_density_arithmetic_matches_oracle(oracle, norb, na, nb):
    """The density kernels' arithmetic (tables, C2 sign convention, D1 from Tab's traces,
    assembly), restated in numpy on the library's hole tables, gives the oracle's pool
    gradient at theta = 0."""
    pool = nw.ucc_pool(norb)
    kind, idx, coef = cuotf.pool_plan(pool.network)
    B = oracle.basis(norb, na, nb)
    rng = np.random.default_rng(norb * 10 + na)
    l, r = rng.normal(size=B.dim), rng.normal(size=B.dim)
    ref = oracle.batchgrad(B, oracle.network(pool.network), np.zeros(pool.network.ngs), l, r)
    got = tdm.emulate_device(B.strings(0, 0), B.strings(0, 1), l, r, norb, kind, idx, coef, cuotf.hole_table)
    assert np.abs(got - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("norb,na,nb,sms,zcap", [(9, 3, 3, 148, 65535), (12, 3, 2, 148, 65535), (9, 3, 3, 2, 65535),
                                                   (9, 3, 3, 148, 5)])
def test_density_kernel_indexing_emulated(oracle, norb, na, nb, sms, zcap):
    """tab_kernel and pair2_kernel emulated thread by thread (launch grid and K splits of
    the host code, shared-memory fill items, mma.sync m8n8k4 lane fragments, atomic flush
    addresses; every index bounds-checked) give the density tables.  The cases cover
    several output tiles, a zero-padded last K slice, K splits of several hole strings per
    CTA (a GPU of 2 multiprocessors), split beta ranges, and a pair2 grid capped below
    its item count (CTAs looping over several hole strings, as for large nH2)."""
    import _kernel_emu as emu
    pool = nw.ucc_pool(norb)
    kind, idx, coef = cuotf.pool_plan(pool.network)
    B = oracle.basis(norb, na, nb)
    A, Bs = B.strings(0, 0), B.strings(0, 1)
    rng = np.random.default_rng(norb + sms)
    l, r = rng.normal(size=B.dim), rng.normal(size=B.dim)
    tb = {}
    tdm.emulate_device(A, Bs, l, r, norb, kind, idx, coef, cuotf.hole_table, tables_out=tb)
    _, tA = cuotf.hole_table(A, norb, 1)
    _, tB = cuotf.hole_table(Bs, norb, 1)
    C = emu.tab(norb, len(Bs), tA, tB, tb["lt"], tb["rt"], sms=sms)
    assert np.abs(C - tb["C"]).max() <= 1e-13 * np.abs(tb["C"]).max()
    for spin, strs in ((0, A), (1, Bs)):
        _, t2 = cuotf.hole_table(strs, norb, 2)
        C2 = emu.pair2(norb, len(A), len(Bs), t2, tb["lt"], tb["rt"], spin, sms=sms, zcap=zcap)
        ref = tb["C2a" if spin == 0 else "C2b"]
        assert np.abs(C2 - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("norb,na,nb,orbsym,tsym", [(6, 3, 2, [0, 1, 2, 3, 0, 1], 1),
                                                    (7, 3, 3, [0, 1, 2, 3, 0, 1, 2], 2)])
def test_density_gradient_on_symmetry_blocks(oracle, norb, na, nb, orbsym, tsym):
    """A symmetry-blocked basis embedded in the dense array over all alpha and beta strings
    (zeros outside the basis) gives the oracle's pool gradient through the unchanged
    single-block arithmetic, on the library's hole tables of the union string lists."""
    pool = nw.ucc_pool(norb)
    net = pool.network
    net.orbsym = np.asarray(orbsym, np.int64)
    kind, idx, coef = cuotf.pool_plan(net)
    B = oracle.basis(norb, na, nb, orbsym=orbsym, total_sym=tsym, num_irreps=4)
    assert B.num_blocks > 1
    rng = np.random.default_rng(norb + tsym)
    l, r = rng.normal(size=B.dim), rng.normal(size=B.dim)
    ref = oracle.batchgrad(B, oracle.network(net), np.zeros(net.ngs), l, r)
    A, Bs, L = tdm.embed_blocks(B, l)
    _, _, R = tdm.embed_blocks(B, r)
    got = tdm.emulate_device(A, Bs, L.ravel(), R.ravel(), norb, kind, idx, coef, cuotf.hole_table)
    assert np.abs(got - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())
