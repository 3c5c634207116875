"""The reference's known answers on the GPU engine, through the public
Circuit API (and so through the C ABI and the CUDA kernels)."""
import pytest

from harness import bit_index, init_index, ket_circuit, load_kats, oracle_circuit, tol

pytestmark = pytest.mark.gpu
CASES = load_kats()


def eval_ket(case):
    import ket_b200 as K
    c = ket_circuit(case)
    init = case.get("init")
    probs = c.exactProbs(initialState=init)
    for chk in case["checks"]:
        kind = chk[0]
        if kind == "amp":
            idx = bit_index(chk[1])
            a = c.amplitudes([idx], initialState=init)[0]
            assert abs(a.real - chk[2]) < tol(chk[4]), (case["id"], chk, a)
            assert abs(a.imag - chk[3]) < tol(chk[4]), (case["id"], chk, a)
        elif kind == "prob":
            assert abs(probs.get(chk[1], 0.0) - chk[2]) < tol(chk[3]), (case["id"], chk, probs)
        elif kind == "nkeys":
            assert len(probs) == chk[1], (case["id"], probs)
        elif kind == "uniform":
            assert all(abs(v - chk[1]) < tol(chk[2]) for v in probs.values())
        elif kind == "marg":
            m = c.marginals(initialState=init)
            assert abs(m[chk[1]] - chk[2]) < tol(chk[3])
        elif kind == "norm":
            assert abs(sum(probs.values()) - 1.0) < tol(chk[1])
        elif kind == "vqe":
            e = K.vqe(c, [(t[0], t[1]) for t in chk[1]])
            assert abs(e - chk[2]) < tol(chk[3]), (case["id"], e)
        elif kind == "expect":
            e = c.expectation(chk[1])
            assert abs(e - chk[2]) < tol(chk[3]), (case["id"], e)
    return c


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_kat_gpu(case):
    import numpy as np
    from oracle import oracle as O
    c = eval_ket(case)
    # and the full state against the oracle's sparse (reference) simulation
    st = oracle_circuit(case).simulate(init=init_index(case), mode=O.SPARSE)
    want = st.dense()
    got = c.statevector_array(initialState=case.get("init"))
    assert np.max(np.abs(got - want)) < 1e-12
