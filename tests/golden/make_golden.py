"""Generate the golden MVP fixtures in this folder.

Run in a container where the TenCirPauli reference checkout is present:

    python tests/golden/make_golden.py /path/to/TenCirPauli

The expected outputs come from the reference's own independent dense oracle
``tests/reference.py`` (Kronecker products of the Pauli matrices, qubit 0 as
the most significant bit), imported from the reference checkout, and from the
fixed vectors written in the reference's tests.  The inputs replicate the
random streams of the reference tests that pin the MVP path:

* ``tests/test_hamiltonian.py:15-24,51-68``  make_operator(n), n in {0,1,2,5}
* ``tests/test_hamiltonian.py:126-147``       random complex differential, n=0..6
* ``tests/test_hamiltonian.py:71-77``         first/last qubit ordering
* ``tests/test_native_abi.py:84-120``         H = 2Z + I, apply([1,2]) == [3,-2]
* ``tests/test_pauli_operator.py:23-30,223-238`` canonical order / aggregation
* ``crates/tencir-pauli-core/src/tests.rs:25-37,121-158`` mvp_test_operator
* ``tests/test_integral_ingestion.py:11-38``   spin-orbital integrals -> the
  expected fermionic terms (the 1/2 two-body factor, index order, constant)

Only the fixtures are committed; the tests never read the reference checkout.
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _codes_from_string(word: str) -> tuple:
    return tuple("IXYZ".index(ch) for ch in word)


def _dense_field(n: int, dense: np.ndarray) -> dict:
    """The reference's dense matrix itself, kept for n <= 6 (pins dense/COO/CSR)."""
    return {"dense": np.asarray(dense, dtype=np.complex128)} if n <= 6 else {}


def main(reference_root: str) -> None:
    sys.path.insert(0, os.path.join(reference_root, "tests"))
    from reference import dense_operator  # the reference's independent oracle

    out = {}

    # make_operator (test_hamiltonian.py:15-24) for n in (0, 1, 2, 5)
    for n in (0, 1, 2, 5):
        structures = [
            tuple((index + qubit) % 4 for qubit in range(n))
            for index in range(min(10, 4**n))
        ]
        coefficients = [complex(index + 1, -index / 3) for index in range(len(structures))]
        state = np.arange(1 << n, dtype=np.float64) + 1j * np.arange(1 << n)
        dense = dense_operator(n, structures, coefficients)
        out[f"make_operator_{n}"] = dict(
            nqubits=np.int64(n),
            codes=np.asarray(structures, dtype=np.uint8).reshape(len(structures), n),
            coefficients=np.asarray(coefficients, dtype=np.complex128),
            state=state,
            expected=dense @ state,
            **_dense_field(n, dense),
        )

    # random complex differential (test_hamiltonian.py:126-147), same RNG stream
    rng = np.random.default_rng(20260801)
    for n in range(7):
        structures = tuple(
            tuple(int(value) for value in rng.integers(0, 4, size=n)) for _ in range(24)
        )
        coefficients = tuple(
            complex(float(re), float(im)) for re, im in rng.normal(size=(24, 2))
        )
        state = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
        dense = dense_operator(n, structures, coefficients)
        out[f"random_differential_{n}"] = dict(
            nqubits=np.int64(n),
            codes=np.asarray(structures, dtype=np.uint8).reshape(24, n),
            coefficients=np.asarray(coefficients, dtype=np.complex128),
            state=state,
            expected=dense @ state,
            **_dense_field(n, dense),
        )

    # qubit ordering (test_hamiltonian.py:71-77): one term on qubit 0 or qubit 2
    for code in (1, 2, 3):
        for name, codes in (("first", (code, 0, 0)), ("last", (0, 0, code))):
            dense = dense_operator(3, (codes,), (1.0,))
            state = np.arange(8, dtype=np.float64) + 0.5j * np.arange(8)[::-1]
            out[f"ordering_{name}_{code}"] = dict(
                nqubits=np.int64(3),
                codes=np.asarray([codes], dtype=np.uint8),
                coefficients=np.asarray([1.0], dtype=np.complex128),
                state=state,
                expected=dense @ state,
                **_dense_field(3, dense),
            )

    # ABI fixed vector (test_native_abi.py:84-120): H = 2Z + I on one qubit
    out["abi_fixed"] = dict(
        nqubits=np.int64(1),
        codes=np.asarray([_codes_from_string("Z"), _codes_from_string("I")], dtype=np.uint8),
        coefficients=np.asarray([2.0, 1.0], dtype=np.complex128),
        state=np.asarray([1.0, 2.0], dtype=np.complex128),
        expected=np.asarray([3.0, -2.0], dtype=np.complex128),
    )

    # mvp_test_operator (tests.rs:25-37) at (1 qubit, 1 term) and (10, 64),
    # with the states of tests.rs:123,140-143
    for n, t in ((1, 1), (10, 64)):
        structures = [
            tuple(int(bool(mask & (1 << q))) for q in range(n)) for mask in range(t)
        ]
        coefficients = [complex(index + 1.0, -index * 0.25) for index in range(t)]
        if n == 1:
            state = np.asarray([3.0 - 2.0j, 5.0 + 4.0j])
        else:
            index = np.arange(1 << n, dtype=np.float64)
            state = index * 0.5 + 1j * (1.0 - index * 0.125)
        dense = dense_operator(n, structures, coefficients)
        out[f"rust_fixture_{n}_{t}"] = dict(
            nqubits=np.int64(n),
            codes=np.asarray(structures, dtype=np.uint8).reshape(t, n),
            coefficients=np.asarray(coefficients, dtype=np.complex128),
            state=state,
            expected=dense @ state,
            **_dense_field(n, dense),
        )

    for name, fields in out.items():
        np.savez(os.path.join(HERE, f"{name}.npz"), **fields)

    # canonicalization known answers written in the reference tests
    np.savez(
        os.path.join(HERE, "canonical_known_answers.npz"),
        # test_pauli_operator.py:23-30
        a_codes=np.asarray(
            [_codes_from_string(w) for w in ("ZX", "II", "ZX", "II")], dtype=np.uint8
        ),
        a_coefficients=np.asarray([1.0, 2.0, -0.25j, -2.0], dtype=np.complex128),
        a_expected_codes=np.asarray([_codes_from_string("ZX")], dtype=np.uint8),
        a_expected_coefficients=np.asarray([1.0 - 0.25j], dtype=np.complex128),
        # test_pauli_operator.py:223-238
        b_codes=np.asarray([[3, 1], [0, 0], [3, 1]], dtype=np.uint8),
        b_coefficients=np.asarray([1.0, 2.0, -0.25j], dtype=np.complex128),
        b_expected_codes=np.asarray([[0, 0], [3, 1]], dtype=np.uint8),
        b_expected_coefficients=np.asarray([2.0, 1.0 - 0.25j], dtype=np.complex128),
    )
    write_integral_known_answer()
    print(f"wrote {len(out) + 2} fixtures to {HERE}")


# Fermionic ladder actions in the term arrays below.
CREATE, ANNIHILATE = 1, 0


def write_integral_known_answer() -> None:
    """tests/test_integral_ingestion.py:11-38: FermionOperator.from_integrals
    of these spin-orbital integrals equals the listed fermionic terms (one-body
    h_pq a+_p a_q, two-body 1/2 g_pqrs a+_p a+_q a_s a_r, constant kept).  The
    terms are stored as (mode, action) rows padded with -1."""
    one_body = np.array([[1.0, 0.2], [0.2, -0.4]], dtype=np.float64)
    two_body = np.zeros((2, 2, 2, 2), dtype=np.float64)
    two_body[0, 1, 0, 1] = 2.0
    terms = [
        ((), 1.25),
        (((0, CREATE), (0, ANNIHILATE)), 1.0),
        (((0, CREATE), (1, ANNIHILATE)), 0.2),
        (((1, CREATE), (0, ANNIHILATE)), 0.2),
        (((1, CREATE), (1, ANNIHILATE)), -0.4),
        (((0, CREATE), (1, CREATE), (1, ANNIHILATE), (0, ANNIHILATE)), 1.0),
    ]
    ops = np.full((len(terms), 4, 2), -1, dtype=np.int64)
    for i, (word, _) in enumerate(terms):
        for j, (mode, action) in enumerate(word):
            ops[i, j] = (mode, action)
    np.savez(
        os.path.join(HERE, "integral_known_answer.npz"),
        one_body=one_body,
        two_body=two_body,
        constant=np.float64(1.25),
        term_ops=ops,
        term_coefficients=np.asarray([c for _, c in terms], dtype=np.complex128),
    )


if __name__ == "__main__":
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("reference_root", help="path of the TenCirPauli reference checkout")
    parser.add_argument("--only-integrals", action="store_true",
                        help="write only the integral known answer (its data is literal, no checkout is read)")
    ns = parser.parse_args()
    if ns.only_integrals:
        write_integral_known_answer()
    else:
        main(ns.reference_root)
