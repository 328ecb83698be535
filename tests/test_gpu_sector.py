"""GPU parity tests of the U(1) sector plans (``include/tcp_sector.h``)
against the oracle (``oracle/u1_oracle.c``), the reference's own sector test
cases, and -- at the full 4x6 J1-J2 size -- the full-space device plan.

Tolerances: complex128 results within rtol = atol = 1e-12 of the oracle (the
reference's sector tests use ``assert_allclose`` defaults on small cases and
the MVP tests 1e-12); CSR columns are bit-exact and CSR values, which the
oracle and the kernel sum in the same order from zero, are bit-exact too;
complex64 applies within a norm-relative 2e-6 of the FP64 oracle.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("CUDA device required", allow_module_level=True)

from tencirpauli_b200 import PauliOperator, U1Sector, workloads  # noqa: E402

FP64_RTOL = 1e-12
C64_NORM_RTOL = 2e-6


def _local(n: int, code: str, *qubits: int) -> str:
    s = ["I"] * n
    for q in qubits:
        s[q] = code
    return "".join(s)


def _conserving(n: int, seed: int, extra_exchanges: int = 0) -> PauliOperator:
    rng = np.random.default_rng(seed)
    terms = [("I" * n, complex(rng.normal(), rng.normal()))]
    for q in range(n - 1):
        h = complex(rng.normal(), rng.normal())
        terms += [(_local(n, "X", q, q + 1), h), (_local(n, "Y", q, q + 1), h)]
    for q in range(n):
        terms.append((_local(n, "Z", q), complex(rng.normal(), rng.normal())))
    used = {(q, q + 1) for q in range(n - 1)}
    for _ in range(extra_exchanges):
        a, b = sorted(int(v) for v in rng.choice(n, size=2, replace=False))
        if (a, b) in used:  # one word per x mask: no cancelling sums (see the leakage test)
            continue
        used.add((a, b))
        h = complex(rng.normal(), 0.5 * rng.normal())
        mid = "Z" * (b - a - 1) if rng.random() < 0.5 else "I" * (b - a - 1)
        terms += [("I" * a + "X" + mid + "X" + "I" * (n - b - 1), h), ("I" * a + "Y" + mid + "Y" + "I" * (n - b - 1), h)]
        c, d = sorted(int(v) for v in rng.choice(n, size=2, replace=False))
        terms.append((_local(n, "Z", c, d), complex(rng.normal(), 0.0)))
    return PauliOperator.from_terms(n, terms)


def _oracle_apply(op: PauliOperator, k: int, state: np.ndarray) -> np.ndarray:
    return oracle.u1_apply(op.nqubits, k, op.x_words, op.z_words, op.coefficients, state)


def _close(got: np.ndarray, ref: np.ndarray) -> None:
    scale = float(np.max(np.abs(ref))) if ref.size else 0.0
    np.testing.assert_allclose(got, ref, rtol=FP64_RTOL, atol=FP64_RTOL * max(scale, 1e-300))


@pytest.mark.parametrize("n", [1, 2, 5, 8, 11])
@pytest.mark.parametrize("storage", ["lazy", "eager"])
def test_every_particle_number_matches_oracle(n: int, storage: str) -> None:
    op = _conserving(n, seed=n, extra_exchanges=n // 2)
    rng = np.random.default_rng(3 * n)
    for k in range(n + 1):
        restricted = op.restrict_charge(U1Sector(n, k), storage=storage)
        plan = restricted.mvp_plan(storage=storage)
        dim = math.comb(n, k)
        state = rng.normal(size=dim) + 1j * rng.normal(size=dim)
        ref = _oracle_apply(op, k, state)
        _close(plan.apply(state), ref)
        _close(restricted.apply(state), ref)
        out = np.full(dim, 9.0 + 4.0j)
        plan.apply_into(np.ascontiguousarray(state), out, max_bytes=0)
        np.testing.assert_array_equal(out, plan.apply(state))


@pytest.mark.parametrize("n,k", [(14, 7), (16, 5), (16, 11), (18, 9)])
def test_medium_sectors_and_complement_ranks_match_oracle(n: int, k: int) -> None:
    op = _conserving(n, seed=100 + n + k, extra_exchanges=3 * n)
    plan = op.restrict_charge(U1Sector(n, k)).mvp_plan()
    assert plan._native_plan.info.complement == (1 if k > n - k else 0)
    rng = np.random.default_rng(n * k)
    dim = math.comb(n, k)
    state = rng.normal(size=dim) + 1j * rng.normal(size=dim)
    _close(plan.apply(state), _oracle_apply(op, k, state))


@pytest.mark.parametrize("n,k", [(40, 2), (64, 2), (64, 63), (48, 3)])
def test_wide_single_word_sectors_use_64_bit_states(n: int, k: int) -> None:
    terms = []
    for q in range(n - 1):
        terms += [(_local(n, "X", q, q + 1), 0.5 + 0.1j * (q % 3)), (_local(n, "Y", q, q + 1), 0.5 + 0.1j * (q % 3))]
    terms += [(_local(n, "Z", q), 0.01 * q) for q in range(0, n, 7)]
    op = PauliOperator.from_terms(n, terms)
    plan = op.restrict_charge(U1Sector(n, k), storage="eager").mvp_plan(storage="eager")
    dim = math.comb(n, k)
    rng = np.random.default_rng(n + k)
    state = rng.normal(size=dim) + 1j * rng.normal(size=dim)
    _close(plan.apply(state), _oracle_apply(op, k, state))
    indptr, cols, vals = oracle.u1_csr(n, k, op.x_words, op.z_words, op.coefficients)
    assert plan.transition_count == len(cols)


def test_reference_projection_case_compile_dispatch_and_eigsh() -> None:
    # tests/test_symmetry.py:185-226 and tests/test_scipy_linear_operator.py:104-124
    op = PauliOperator.from_terms(3, [("XXI", 0.5), ("YYI", 0.5), ("IZZ", -0.25), ("ZII", 0.1)])
    restricted = op.restrict_charge(U1Sector(3, 1))
    with pytest.warns(DeprecationWarning, match="restrict_charge"):
        alias = op.restrict_u1(U1Sector(3, 1))
    state = np.asarray([1.0, 2.0, 3.0], np.complex128)
    ref = _oracle_apply(op, 1, state)
    _close(restricted.apply(state), ref)
    _close(restricted.mvp_plan().apply(state), ref)
    np.testing.assert_array_equal(alias.apply(state), restricted.apply(state))
    dense = restricted.dense()
    _close(dense @ state, ref)
    coo = restricted.coo()
    from_coo = np.zeros_like(dense)
    from_coo[coo.row.astype(np.int64), coo.column.astype(np.int64)] = coo.data
    np.testing.assert_array_equal(from_coo, dense)
    csr = restricted.compile("csr")
    np.testing.assert_array_equal(csr.to_scipy().toarray(), dense)
    assert restricted.compile("native_mvp").storage == "lazy"
    assert restricted.compile("native_mvp", storage="eager").storage == "eager"
    with pytest.raises(ValueError, match="target must be one of"):
        restricted.compile("backend_mvp")

    op4 = PauliOperator.from_terms(4, [("ZIII", 0.5), ("IZII", -0.5), ("XXII", 0.25), ("YYII", 0.25)])
    r4 = op4.restrict_charge(U1Sector(4, 2))
    plan4 = r4.mvp_plan()
    linear = plan4.to_scipy_linear_operator()
    vector = np.arange(6, dtype=np.float64) + 1j * np.arange(6, dtype=np.float64)
    _close(linear.matvec(vector), r4.dense() @ vector)
    from scipy.sparse.linalg import eigsh

    values, _ = eigsh(linear, k=1, which="SA")
    np.testing.assert_allclose(values[0], np.linalg.eigvalsh(r4.dense())[0], atol=1e-12)


def test_csr_is_bit_exact_against_the_oracle_csr() -> None:
    op = _conserving(9, seed=42, extra_exchanges=6)
    for k in (0, 3, 4, 6, 9):
        restricted = op.restrict_charge(U1Sector(9, k), storage="eager")
        csr = restricted.csr()
        indptr, cols, vals = oracle.u1_csr(9, k, op.x_words, op.z_words, op.coefficients)
        np.testing.assert_array_equal(csr.indptr, indptr)
        np.testing.assert_array_equal(csr.indices, cols)
        assert csr.data.tobytes() == vals.tobytes()
        assert restricted.mvp_plan(storage="eager").transition_count == len(cols)


def test_leakage_errors_match_the_oracle() -> None:
    # eager restriction scans sources in order; the lowest leaking source is named
    leak = PauliOperator.from_terms(3, [("XII", 1.0)])
    with pytest.raises(oracle.OracleLeakage) as ref:
        _oracle_apply(leak, 1, np.ones(3, np.complex128))
    with pytest.raises(ValueError, match="U\\(1\\) sector leakage") as got:
        leak.restrict_charge(U1Sector(3, 1), storage="eager")
    assert f"source index {ref.value.source}" in str(got.value)
    assert f"destination weight {ref.value.weight}" in str(got.value)
    # XX alone keeps weight 1 but not weight 0: eager accepts k = 1, rejects k = 0;
    # lazy restriction applies the global commutator rule and rejects both
    xx = PauliOperator.from_terms(2, [("XX", 1.0)])
    eager = xx.restrict_charge(U1Sector(2, 1), storage="eager")
    _close(eager.apply(np.asarray([1.0, 2.0], np.complex128)), _oracle_apply(xx, 1, np.asarray([1.0, 2.0], np.complex128)))
    with pytest.raises(ValueError, match="source index 0: expected particle number 0, got destination weight 2"):
        xx.restrict_charge(U1Sector(2, 0), storage="eager")
    with pytest.raises(ValueError, match="exactly conserved operator"):
        xx.restrict_charge(U1Sector(2, 1))
    # X2 (1 + Z3) / 2 leaks only from sources with qubit 3 clear: the first is
    # |0110> (sector index 2), sent to weight 1
    mixed = PauliOperator.from_terms(4, [("XXII", 0.5), ("YYII", 0.5), ("IIXI", 0.5), ("IIXZ", 0.5)])
    with pytest.raises(oracle.OracleLeakage) as ref2:
        _oracle_apply(mixed, 2, np.ones(6, np.complex128))
    assert (ref2.value.source, ref2.value.weight) == (2, 1)
    with pytest.raises(ValueError, match="source index 2: expected particle number 2, got destination weight 1"):
        mixed.restrict_charge(U1Sector(4, 2), storage="eager")


def test_rounding_leak_of_an_aggregated_group_is_reported_like_the_reference() -> None:
    """XIX + XZX - YIY - YZY conserves the particle number exactly, but its
    x-mask group sums ((h2 + h1 s) - h2) - h1 s in canonical term order, which
    rounds to a tiny nonzero value on sources whose two flipped qubits agree.
    The reference's aggregate_source then reports SectorLeakage; both
    storages report it here at build time, naming the oracle's source."""
    h1, h2 = 0.1 + 0.2j, 0.7 - 0.3j
    op = PauliOperator.from_terms(
        4, [("XIXI", h2), ("XZXI", h1), ("YIYI", h2), ("YZYI", h1), ("ZIII", 0.4)]
    )
    assert op.conserves_particle_number()
    for k in range(5):
        try:
            _oracle_apply(op, k, np.ones(math.comb(4, k), np.complex128))
        except oracle.OracleLeakage as ref:
            for storage in ("lazy", "eager"):
                with pytest.raises(ValueError, match=f"source index {ref.source}: .*weight {ref.weight}"):
                    op.restrict_charge(U1Sector(4, k), storage=storage)
        else:
            restricted = op.restrict_charge(U1Sector(4, k))
            state = np.arange(math.comb(4, k), dtype=np.complex128) + 1j
            _close(restricted.apply(state), _oracle_apply(op, k, state))


def test_complex64_multi_rhs_and_diagonal_on_the_device() -> None:
    n, k = 16, 8
    op = _conserving(n, seed=5, extra_exchanges=20)
    plan = op.restrict_charge(U1Sector(n, k)).mvp_plan()
    dim = plan.dimension
    xs = workloads.random_state_device(n, seed=9, nrhs=3, length=dim)
    ys = torch.empty_like(xs)
    plan.apply_device(xs, ys)
    torch.cuda.synchronize()
    for v in range(3):
        ref = _oracle_apply(op, k, xs[v].cpu().numpy())
        _close(ys[v].cpu().numpy(), ref)
    x64 = xs.to(torch.complex64)
    y64 = torch.empty_like(x64)
    plan.apply_device(x64, y64)
    torch.cuda.synchronize()
    rel = torch.linalg.vector_norm(y64.to(torch.complex128) - ys) / torch.linalg.vector_norm(ys)
    assert float(rel) <= C64_NORM_RTOL
    diag = torch.empty(dim, dtype=torch.complex128, device="cuda")
    plan.diagonal_device(diag)
    torch.cuda.synchronize()
    dense = op.restrict_charge(U1Sector(n, k), storage="eager")
    indptr, cols, vals = oracle.u1_csr(n, k, op.x_words, op.z_words, op.coefficients)
    ref_diag = np.zeros(dim, np.complex128)
    for r in range(dim):
        sel = cols[indptr[r] : indptr[r + 1]] == r
        if np.any(sel):
            ref_diag[r] = vals[indptr[r] : indptr[r + 1]][sel][0]
    np.testing.assert_array_equal(diag.cpu().numpy(), ref_diag)
    del dense
    plan._native_plan.device_status()


def test_many_terms_run_from_global_memory_and_match_oracle() -> None:
    """More term data than the shared-memory staging budget: the
    global-memory variant.  Every hopping pair carries many Z strings; the
    coefficients are dyadic so that the x-mask groups cancel exactly on
    sources outside the sector (no rounding leak)."""
    n, k = 14, 6
    rng = np.random.default_rng(78)
    terms = [(_local(n, "Z", q), float(rng.integers(-8, 9)) / 8) for q in range(n)]
    for a in range(n):
        for b in range(a + 1, n):
            others = [q for q in range(n) if q not in (a, b)]
            for _ in range(80):
                zs = set(int(q) for q in rng.choice(others, size=int(rng.integers(0, 5)), replace=False))
                h = complex(int(rng.integers(-16, 17)), int(rng.integers(-16, 17))) / 16
                for code in "XY":
                    w = ["Z" if q in zs else "I" for q in range(n)]
                    w[a] = w[b] = code
                    terms.append(("".join(w), h))
    op = PauliOperator.from_terms(n, terms)
    plan = op.restrict_charge(U1Sector(n, k)).mvp_plan()
    assert plan._native_plan.info.tables_in_shared == 0
    state = rng.normal(size=plan.dimension) + 1j * rng.normal(size=plan.dimension)
    _close(plan.apply(state), _oracle_apply(op, k, state))
    x64 = torch.from_numpy(state.astype(np.complex64)).cuda()
    y64 = torch.empty_like(x64)
    plan.apply_device(x64, y64)
    ref = _oracle_apply(op, k, state.astype(np.complex64).astype(np.complex128))
    got = y64.cpu().numpy().astype(np.complex128)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= C64_NORM_RTOL


def test_single_word_width_boundary_and_the_width_limit() -> None:
    # tests/test_symmetry.py:281-286: n = 64, k = 0 (one state)
    op = PauliOperator.from_terms(64, [("I" * 64, 1.0)])
    restricted = op.restrict_charge(U1Sector(64, 0))
    np.testing.assert_allclose(restricted.apply(np.asarray([2.0 + 3.0j])), [2.0 + 3.0j])
    wide = PauliOperator.from_terms(257, [(_local(257, "X", 3, 4), 0.5), (_local(257, "Y", 3, 4), 0.5)])
    with pytest.raises(OverflowError, match="at most 256 qubits"):
        wide.restrict_charge(U1Sector(257, 1))


def _hopping(n: int, coefficient: complex = 0.5) -> PauliOperator:
    terms = []
    for q in range(n - 1):
        terms += [(_local(n, "X", q, q + 1), coefficient), (_local(n, "Y", q, q + 1), coefficient)]
    return PauliOperator.from_terms(n, terms)


@pytest.mark.parametrize("n,k", [(63, 1), (64, 1), (65, 2), (65, 63), (127, 1), (128, 2), (129, 2), (256, 1)])
def test_wide_sector_restriction_matches_the_oracle(n: int, k: int) -> None:
    # the cases of tests/test_u1.py:125-154 of the reference
    op = _hopping(n)
    restricted = op.restrict_charge(U1Sector(n, k), storage="eager")
    indptr, cols, vals = oracle.u1_csr(n, k, op.x_words, op.z_words, op.coefficients)
    csr = restricted.csr()
    np.testing.assert_array_equal(csr.indptr, indptr)
    np.testing.assert_array_equal(csr.indices, cols)
    assert csr.data.tobytes() == vals.tobytes()
    rng = np.random.default_rng(n + k)
    state = rng.normal(size=restricted.dimension) + 1j * rng.normal(size=restricted.dimension)
    ref = _oracle_apply(op, k, state)
    _close(restricted.apply(state), ref)
    _close(op.restrict_charge(U1Sector(n, k)).mvp_plan().apply(state), ref)


def test_wide_sector_complex_hopping_across_a_word_boundary_and_leakage() -> None:
    # tests/test_u1.py:157-199 of the reference: qubits 63 and 64 straddle two words
    n = 65
    coefficient = 0.7 + 0.2j
    op = PauliOperator.from_terms(n, [(_local(n, "X", 63, 64), coefficient), (_local(n, "Y", 63, 64), coefficient),
                                      (_local(n, "Z", 64), 0.3)])
    restricted = op.restrict_charge(U1Sector(n, 1), storage="eager")
    indptr, cols, vals = oracle.u1_csr(n, 1, op.x_words, op.z_words, op.coefficients)
    csr = restricted.csr()
    np.testing.assert_array_equal(csr.indices, cols)
    assert csr.data.tobytes() == vals.tobytes()
    plan = restricted.mvp_plan(storage="eager")
    diag = torch.empty(plan.dimension, dtype=torch.complex128, device="cuda")
    plan.diagonal_device(diag)
    torch.cuda.synchronize()
    dense = restricted.dense()
    np.testing.assert_array_equal(diag.cpu().numpy(), np.diag(dense))
    leaking = PauliOperator.from_terms(129, [(_local(129, "X", 64), 1.0)])
    with pytest.raises(ValueError, match=r"U\(1\) sector leakage"):
        leaking.restrict_charge(U1Sector(129, 1))
    with pytest.raises(ValueError, match="source index 0: expected particle number 1, got destination weight 2"):
        leaking.restrict_charge(U1Sector(129, 1), storage="eager")
    ok = PauliOperator.from_terms(129, [(_local(129, "X", 63, 64), 0.5), (_local(129, "Y", 63, 64), 0.5)])
    assert ok.restrict_charge(U1Sector(129, 1)).dimension == 129


def test_j1j2_4x6_half_filling_equals_the_full_space_plan() -> None:
    """Full size (D = C(24, 12) = 2,704,156): the sector apply equals the
    full-space device plan applied to the embedded state and read back on the
    sector, and the restricted operator is Hermitian."""
    op = PauliOperator.from_code_arrays(*workloads.j1j2_periodic(4, 6, 1.0, 0.5))
    n, k = 24, 12
    plan = op.restrict_charge(U1Sector(n, k)).mvp_plan()
    assert plan.dimension == math.comb(n, k)
    ints = np.arange(1 << n, dtype=np.int64)
    weights = np.bitwise_count(ints.astype(np.uint64))
    basis = torch.from_numpy(ints[weights == k]).cuda()  # ascending = sector order
    assert basis.numel() == plan.dimension
    x = workloads.random_state_device(n, seed=21, length=plan.dimension)
    y = torch.empty_like(x)
    plan.apply_device(x, y)
    full = op.native_mvp_plan()
    xf = torch.zeros(1 << n, dtype=torch.complex128, device="cuda")
    xf[basis] = x
    yf = torch.empty_like(xf)
    full.apply_device(xf, yf)
    torch.cuda.synchronize()
    ref = yf[basis]
    err = torch.linalg.vector_norm(y - ref) / torch.linalg.vector_norm(ref)
    assert float(err) <= FP64_RTOL
    assert float(torch.linalg.vector_norm(yf) - torch.linalg.vector_norm(ref)) <= 1e-12 * float(torch.linalg.vector_norm(ref))
    a = workloads.random_state_device(n, seed=22, length=plan.dimension)
    ha = torch.empty_like(a)
    plan.apply_device(a, ha)
    lhs, rhs = complex(torch.vdot(a, y)), complex(torch.vdot(ha, x))
    assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(lhs))
    del xf, yf, ints, weights
    torch.cuda.empty_cache()


def test_davidson_in_the_half_filling_sector_matches_dense() -> None:
    from tencirpauli_b200.davidson import davidson

    op = PauliOperator.from_code_arrays(*workloads.j1j2_periodic(3, 4, 1.0, 0.5))
    restricted = op.restrict_charge(U1Sector(12, 6))
    plan = restricted.mvp_plan()
    ref = np.linalg.eigvalsh(restricted.dense())[:4]
    res = davidson(plan, nev=4, tol=1e-8, seed=2)
    assert res.converged
    np.testing.assert_allclose(res.eigenvalues, ref, atol=1e-9)


def test_large_sector_host_apply_streams_output_chunks_and_matches_device_path() -> None:
    """D = C(26, 13) = 10,400,600: the host entry point runs the sector kernel
    over row ranges and copies each finished range back while the next one
    computes; the result equals the device path bit for bit."""
    op = PauliOperator.from_code_arrays(*workloads.heisenberg_chain(26))
    plan = op.restrict_charge(U1Sector(26, 13)).mvp_plan()
    x = workloads.random_state_device(26, seed=8, length=plan.dimension)
    y = torch.empty_like(x)
    plan.apply_device(x, y)
    torch.cuda.synchronize()
    out = np.full(plan.dimension, np.nan, dtype=np.complex128)
    plan.apply_into(x.cpu().numpy(), out)
    np.testing.assert_array_equal(out, y.cpu().numpy())
    rows = np.sort(np.random.default_rng(2).choice(plan.dimension, size=512, replace=False)).astype(np.uint64)
    ref = oracle.u1_apply_rows(26, 13, op.x_words, op.z_words, op.coefficients, x.cpu().numpy(), rows)
    _close(out[rows.astype(np.int64)], ref)
    del x, y
    torch.cuda.empty_cache()
