"""Writes tests/golden/reference_kats.json: known-answer cases of the
statevector path restated from the reference's own test suite
(dmvjs/ket, src/circuit.test.ts and src/gates.test.ts).

The reference is TypeScript and cannot run in this environment (no Node), so
its golden values come from its tests: each case below cites the test it
restates and carries the same circuit and the same expected value and digit
count (vitest toBeCloseTo(x, d) means |got - x| < 0.5 * 10^-d).

Case format: {"id", "cite", "n", "gates": [[name, qubits, params], ...],
"init": q0-leftmost bitstring or null, "checks": [...]} with checks:
  ["amp", bitstring, re, im, digits]     amplitude()
  ["prob", bitstring, p, digits]         exactProbs()[bitstring]
  ["nkeys", k]                           len(exactProbs())
  ["uniform", p, digits]                 every exactProbs() value
  ["marg", q, p, digits]                 marginals()[q]
  ["vqe", [[coeff, ops], ...], e, digits]
  ["expect", pauli, e, digits]           expectation(pauli)
  ["norm", digits]                       sum of exactProbs() == 1
Run: python tests/golden/make_reference_kats.py
"""
import json
import math
import os

PI = math.pi
S2 = 1 / math.sqrt(2)  # Math.SQRT2 / 2 as the tests write 1 / Math.SQRT2
cases = []


def case(id_, cite, n, gates, checks, init=None):
    cases.append({"id": id_, "cite": cite, "n": n, "gates": gates, "init": init, "checks": checks})


# X / H / Z / S / T / V / rotations (circuit.test.ts:116-230)
case("x_flips", "circuit.test.ts:117-121", 1, [["x", [0], []]], [["prob", "1", 1.0, 10], ["nkeys", 1]])
case("xx_identity", "circuit.test.ts:123-126", 1, [["x", [0], []], ["x", [0], []]], [["prob", "0", 1.0, 10]])
case("hh_identity", "circuit.test.ts:137-140", 1, [["h", [0], []], ["h", [0], []]], [["prob", "0", 1.0, 10]])
case("z_on_zero", "circuit.test.ts:144-147", 1, [["z", [0], []]], [["prob", "0", 1.0, 10]])
case("hzh_is_x", "circuit.test.ts:149-152", 1, [["h", [0], []], ["z", [0], []], ["h", [0], []]], [["prob", "1", 1.0, 10]])
case("ss_on_zero", "circuit.test.ts:156-161", 1, [["s", [0], []], ["s", [0], []]], [["prob", "0", 1.0, 10]])
case("sdg_s", "circuit.test.ts:163-166", 1, [["s", [0], []], ["si", [0], []]], [["prob", "0", 1.0, 10]])
case("tdg_t", "circuit.test.ts:170-173", 1, [["t", [0], []], ["ti", [0], []]], [["prob", "0", 1.0, 10]])
case("tttt", "circuit.test.ts:175-178", 1, [["t", [0], []]] * 4, [["prob", "0", 1.0, 10]])
case("vv_is_x", "circuit.test.ts:182-185", 1, [["v", [0], []], ["v", [0], []]], [["prob", "1", 1.0, 10]])
case("vdg_v", "circuit.test.ts:187-190", 1, [["v", [0], []], ["vi", [0], []]], [["prob", "0", 1.0, 10]])
case("rx_pi", "circuit.test.ts:194-197", 1, [["rx", [0], [PI]]], [["prob", "1", 1.0, 5]])
case("rx_0", "circuit.test.ts:205-208", 1, [["rx", [0], [0.0]]], [["prob", "0", 1.0, 10]])
case("ry_pi", "circuit.test.ts:212-215", 1, [["ry", [0], [PI]]], [["prob", "1", 1.0, 5]])
case("ry_2pi", "circuit.test.ts:217-220", 1, [["ry", [0], [2 * PI]]], [["prob", "0", 1.0, 8]])
case("rz_on_zero", "circuit.test.ts:224-227", 1, [["rz", [0], [PI / 3]]], [["prob", "0", 1.0, 10]])
case("h_rz_pi_h", "circuit.test.ts:229-232", 1, [["h", [0], []], ["rz", [0], [PI]], ["h", [0], []]], [["prob", "1", 1.0, 5]])
# CNOT / SWAP (circuit.test.ts:237-270)
case("cnot_00", "circuit.test.ts:238-241", 2, [["cnot", [0, 1], []]], [["prob", "00", 1.0, 10]])
case("cnot_10", "circuit.test.ts:243-247", 2, [["x", [0], []], ["cnot", [0, 1], []]], [["prob", "11", 1.0, 10]])
case("cnot_cnot", "circuit.test.ts:249-252", 2, [["x", [0], []], ["cnot", [0, 1], []], ["cnot", [0, 1], []]],
     [["prob", "10", 1.0, 10]])
case("swap_10", "circuit.test.ts:256-261", 2, [["x", [0], []], ["swap", [0, 1], []]], [["prob", "01", 1.0, 10]])
case("swap_swap", "circuit.test.ts:263-266", 2, [["x", [0], []], ["swap", [0, 1], []], ["swap", [0, 1], []]],
     [["prob", "10", 1.0, 10]])
# statevector() / amplitude() / probability() (circuit.test.ts:1625-1725)
case("sv_zero", "circuit.test.ts:1626-1630", 1, [], [["amp", "0", 1.0, 0.0, 15], ["nkeys", 1]])
case("sv_h", "circuit.test.ts:1632-1639", 1, [["h", [0], []]],
     [["amp", "0", S2, 0.0, 10], ["amp", "1", S2, 0.0, 10]])
case("sv_x", "circuit.test.ts:1641-1645", 1, [["x", [0], []]], [["amp", "1", 1.0, 0.0, 10], ["amp", "0", 0.0, 0.0, 10]])
case("sv_bell", "circuit.test.ts:1647-1652", 2, [["h", [0], []], ["cnot", [0, 1], []]],
     [["amp", "00", S2, 0.0, 10], ["amp", "11", S2, 0.0, 10], ["amp", "01", 0.0, 0.0, 10],
      ["amp", "10", 0.0, 0.0, 10], ["nkeys", 2]])
case("amp_s1", "circuit.test.ts:1683-1688", 1, [["x", [0], []], ["s", [0], []]], [["amp", "1", 0.0, 1.0, 10]])
case("prob_sum", "circuit.test.ts:1717-1724", 3, [["h", [0], []], ["cnot", [0, 1], []], ["rx", [2], [0.7]]],
     [["norm", 10]])
# exactProbs() (circuit.test.ts:3436-3470)
case("ep_x", "circuit.test.ts:3437-3441", 1, [["x", [0], []]], [["prob", "1", 1.0, 15], ["nkeys", 1]])
case("ep_h", "circuit.test.ts:3443-3447", 1, [["h", [0], []]], [["prob", "0", 0.5, 15], ["prob", "1", 0.5, 15]])
case("ep_bell", "circuit.test.ts:3449-3454", 2, [["h", [0], []], ["cnot", [0, 1], []]],
     [["prob", "00", 0.5, 15], ["prob", "11", 0.5, 15], ["nkeys", 2]])
case("ep_hh", "circuit.test.ts:3456-3460", 1, [["h", [0], []], ["h", [0], []]], [["prob", "0", 1.0, 12], ["nkeys", 1]])
case("ep_h4", "circuit.test.ts:3462-3469", 4, [["h", [q], []] for q in range(4)], [["nkeys", 16], ["uniform", 1 / 16, 14]])
# marginals() (circuit.test.ts:3701-3736)
case("marg_0", "circuit.test.ts:3702-3705", 1, [], [["marg", 0, 0.0, 12]])
case("marg_1", "circuit.test.ts:3707-3710", 1, [["x", [0], []]], [["marg", 0, 1.0, 12]])
case("marg_plus", "circuit.test.ts:3712-3715", 1, [["h", [0], []]], [["marg", 0, 0.5, 12]])
case("marg_bell", "circuit.test.ts:3717-3721", 2, [["h", [0], []], ["cnot", [0, 1], []]],
     [["marg", 0, 0.5, 12], ["marg", 1, 0.5, 12]])
case("marg_x1", "circuit.test.ts:3723-3727", 2, [["x", [1], []]], [["marg", 0, 0.0, 12], ["marg", 1, 1.0, 12]])
for n in (2, 3, 4, 5):
    case(f"marg_h{n}", "circuit.test.ts:3729-3736", n, [["h", [q], []] for q in range(n)],
         [["marg", q, 0.5, 12] for q in range(n)])
# QFT (circuit.test.ts:3856-3930); qft(n) gates are spelled out (algorithms.ts:16-26)


def qft_gates(n):
    g = []
    for j in range(n - 1, -1, -1):
        g.append(["h", [j], []])
        for k in range(j - 1, -1, -1):
            g.append(["cu1", [k, j], [PI / 2 ** (j - k)]])
    for i in range(n // 2):
        g.append(["swap", [i, n - 1 - i], []])
    return g


for n in (2, 3, 4):
    case(f"qft{n}_uniform", "circuit.test.ts:3869-3877", n, qft_gates(n), [["nkeys", 2 ** n], ["uniform", 1 / 2 ** n, 10]])
case("qft3_on_1", "circuit.test.ts:3917-3930", 3, qft_gates(3),
     [["amp", format(k, "03b")[::-1], math.cos(2 * PI * k / 8) / math.sqrt(8), math.sin(2 * PI * k / 8) / math.sqrt(8), 10]
      for k in range(8)], init="100")
case("qft2_roundtrip", "circuit.test.ts:3903-3911", 2,
     [["x", [0], []], ["h", [1], []], ["cu1", [0, 1], [PI / 2]], ["h", [0], []], ["swap", [0, 1], []],
      ["swap", [0, 1], []], ["h", [0], []], ["cu1", [0, 1], [-PI / 2]], ["h", [1], []]],
     [["prob", "10", 1.0, 10]])
# vqe (circuit.test.ts:4060-4141)
case("vqe_z0", "circuit.test.ts:4061-4064", 1, [], [["vqe", [[1, "Z"]], 1.0, 10]])
case("vqe_z1", "circuit.test.ts:4066-4069", 1, [["x", [0], []]], [["vqe", [[1, "Z"]], -1.0, 10]])
case("vqe_xplus", "circuit.test.ts:4071-4074", 1, [["h", [0], []]], [["vqe", [[1, "X"]], 1.0, 10]])
case("vqe_xminus", "circuit.test.ts:4076-4079", 1, [["x", [0], []], ["h", [0], []]], [["vqe", [[1, "X"]], -1.0, 10]])
case("vqe_yplus", "circuit.test.ts:4081-4085", 1, [["rx", [0], [-PI / 2]]], [["vqe", [[1, "Y"]], 1.0, 8]])
case("vqe_ident", "circuit.test.ts:4087-4090", 1, [], [["vqe", [[3.14, "I"]], 3.14, 10]])
case("vqe_zx", "circuit.test.ts:4092-4103", 1, [["ry", [0], [5 * PI / 4]]],
     [["vqe", [[0.5, "Z"], [0.5, "X"]], -math.sqrt(2) / 2, 8]])
case("vqe_zz00", "circuit.test.ts:4105-4108", 2, [], [["vqe", [[1, "ZZ"]], 1.0, 10]])
case("vqe_zz01", "circuit.test.ts:4110-4113", 2, [["x", [0], []]], [["vqe", [[1, "ZZ"]], -1.0, 10]])
case("vqe_zz_bell", "circuit.test.ts:4115-4118", 2, [["h", [0], []], ["cnot", [0, 1], []]], [["vqe", [[1, "ZZ"]], 1.0, 8]])
case("vqe_xii_0", "circuit.test.ts:4120-4122", 3, [], [["vqe", [[1, "XII"]], 0.0, 10]])
case("vqe_xii_plus", "circuit.test.ts:4124-4126", 3, [["h", [2], []]], [["vqe", [[1, "XII"]], 1.0, 10]])
case("vqe_skip_tiny", "circuit.test.ts:4132-4135", 1, [], [["vqe", [[1e-20, "Z"], [2, "I"]], 2.0, 10]])
case("vqe_lower", "circuit.test.ts:4137-4143", 1, [["x", [0], []]], [["vqe", [[1, "z"]], -1.0, 10]])
# expectation() (circuit.test.ts:7064-7099; docstring examples circuit.ts:3720-3726)
case("exp_z0", "circuit.ts:3722", 1, [], [["expect", "Z", 1.0, 12]])
case("exp_z1", "circuit.ts:3723", 1, [["x", [0], []]], [["expect", "Z", -1.0, 12]])
case("exp_xplus", "circuit.ts:3724", 1, [["h", [0], []]], [["expect", "X", 1.0, 12]])
case("exp_bell_zz", "circuit.ts:3725", 2, [["h", [0], []], ["cnot", [0, 1], []]], [["expect", "ZZ", 1.0, 12]])
case("exp_y", "circuit.test.ts:4081-4085 (Y eigenstate)", 1, [["rx", [0], [-PI / 2]]], [["expect", "Y", 1.0, 10]])
# initialState (circuit.test.ts:5603-5622)
case("init_01", "circuit.test.ts:5604-5609", 2, [["x", [0], []]], [["amp", "11", 1.0, 0.0, 10]], init="01")
case("init_cnot_11", "circuit.test.ts:5619-5622", 2, [["cnot", [0, 1], []]], [["prob", "10", 1.0, 10]], init="11")
case("init_h1", "circuit.test.ts:5611-5617", 1, [["h", [0], []]], [["amp", "0", S2, 0.0, 10], ["amp", "1", -S2, 0.0, 10]],
     init="1")
# normalisation and self-inverse gates (circuit.test.ts:6763-6803)
H2 = [[S2, 0.0, S2, 0.0], [S2, 0.0, -S2, 0.0]]  # unitary() rows as re,im pairs
for cid, n, g in [
    ("h", 1, [["h", [0], []]]),
    ("rx123", 1, [["rx", [0], [1.23]]]),
    ("bell", 2, [["h", [0], []], ["cnot", [0, 1], []]]),
    ("swap_sup", 2, [["h", [0], []], ["swap", [0, 1], []]]),
    ("xx_pi4", 2, [["xx", [0, 1], [PI / 4]]]),
    ("ghz3", 3, [["h", [0], []], ["cnot", [0, 1], []], ["cnot", [1, 2], []]]),
    ("toffoli_sup", 3, [["h", [0], []], ["h", [1], []], ["ccx", [0, 1, 2], []]]),
    ("csrswap", 3, [["h", [1], []], ["csrswap", [0, 1, 2], []]]),
    ("unitary_h", 1, [["unitary", [0], H2]]),
]:
    case(f"norm_{cid}", "circuit.test.ts:6763-6775", n, g, [["norm", 13]])
for g in ("x", "y", "z", "h"):
    case(f"self_inverse_{g}", "circuit.test.ts:6786-6789", 1, [[g, [0], []], [g, [0], []]], [["prob", "0", 1.0, 14]])
case("self_inverse_cnot", "circuit.test.ts:6792", 2, [["x", [0], []], ["cnot", [0, 1], []], ["cnot", [0, 1], []]],
     [["prob", "10", 1.0, 14]])
case("self_inverse_swap", "circuit.test.ts:6793", 2, [["x", [0], []], ["swap", [0, 1], []], ["swap", [0, 1], []]],
     [["prob", "10", 1.0, 14]])
case("self_inverse_cz", "circuit.test.ts:6794", 2, [["x", [0], []], ["cz", [0, 1], []], ["cz", [0, 1], []]],
     [["prob", "10", 1.0, 14]])
case("self_inverse_ccx", "circuit.test.ts:6795", 3, [["x", [0], []], ["x", [1], []], ["ccx", [0, 1, 2], []], ["ccx", [0, 1, 2], []]],
     [["prob", "110", 1.0, 14]])
case("self_inverse_cswap", "circuit.test.ts:6796", 3,
     [["x", [0], []], ["x", [1], []], ["cswap", [0, 1, 2], []], ["cswap", [0, 1, 2], []]], [["prob", "110", 1.0, 14]])
case("self_inverse_bell", "circuit.test.ts:6799-6801", 2,
     [["h", [0], []], ["cnot", [0, 1], []], ["cnot", [0, 1], []], ["h", [0], []]], [["prob", "00", 1.0, 14]])
# Toffoli / Fredkin / C-sqrt(iSWAP) (circuit.test.ts:1283-1440)
case("ccx_nonadjacent", "circuit.test.ts:1337-1340", 7, [["x", [0], []], ["x", [3], []], ["ccx", [0, 3, 6], []]],
     [["prob", "1001001", 1.0, 10]])
case("ccx_phase_kickback", "circuit.test.ts:1329-1334", 3,
     [["x", [0], []], ["x", [1], []], ["x", [2], []], ["h", [2], []], ["ccx", [0, 1, 2], []], ["h", [2], []]],
     [["prob", "111", 1.0, 10]])
case("ccx_11", "circuit.test.ts:1283-1296", 3, [["x", [0], []], ["x", [1], []], ["ccx", [0, 1, 2], []]], [["prob", "111", 1.0, 10]])
case("ccx_10", "circuit.test.ts:1283-1296", 3, [["x", [0], []], ["ccx", [0, 1, 2], []]], [["prob", "100", 1.0, 10]])
case("cswap_on", "circuit.test.ts:1344-1357", 3, [["x", [0], []], ["x", [1], []], ["cswap", [0, 1, 2], []]],
     [["prob", "101", 1.0, 10]])
case("cswap_off", "circuit.test.ts:1344-1357", 3, [["x", [1], []], ["cswap", [0, 1, 2], []]], [["prob", "010", 1.0, 10]])
case("csrswap", "statevector.ts:170-207", 3, [["x", [0], []], ["x", [2], []], ["csrswap", [0, 1, 2], []]],
     [["amp", "101", S2, 0.0, 12], ["amp", "110", 0.0, S2, 12]])
# IonQ native / two-qubit interaction gates (gates.ts identities exercised in gates.test.ts)
case("ms00", "gates.ts:186-190", 2, [["ms", [0, 1], [0.0, 0.0]]], [["prob", "00", 0.5, 12], ["prob", "11", 0.5, 12]])
case("xx_pi2", "gates.ts:95-97", 2, [["xx", [0, 1], [PI / 2]]], [["amp", "00", S2, 0.0, 12], ["amp", "11", 0.0, -S2, 12]])
case("iswap_10", "gates.ts:155-156", 2, [["x", [0], []], ["iswap", [0, 1], []]], [["amp", "01", 0.0, 1.0, 12]])
case("gpi0_is_x", "gates.ts:160-163", 1, [["gpi", [0], [0.0]]], [["prob", "1", 1.0, 12]])
case("gpi2_0_is_rx", "gates.ts:173-176", 1, [["gpi2", [0], [0.0]]], [["amp", "0", S2, 0.0, 12], ["amp", "1", 0.0, -S2, 12]])
case("u3_h", "gates.ts:63-65", 1, [["u3", [0], [PI / 2, 0.0, PI]]], [["amp", "0", S2, 0.0, 12], ["amp", "1", S2, 0.0, 12]])
# QAOA 4-cycle (circuit.test.ts:6373-6421): p=1 expected cut above the 2.0 random baseline
case("qaoa_c4_hamiltonian", "circuit.test.ts:6373-6421", 4,
     [["h", [q], []] for q in range(4)],
     [["vqe", [[2.0, "IIII"], [-0.5, "IIZZ"], [-0.5, "IZZI"], [-0.5, "ZZII"], [-0.5, "ZIIZ"]], 2.0, 12]])

if __name__ == "__main__":
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")
    with open(out, "w") as f:
        json.dump({"source": "dmvjs/ket src/circuit.test.ts, src/gates.test.ts (restated)", "cases": cases}, f, indent=1)
    print(f"wrote {len(cases)} cases to {out}")
