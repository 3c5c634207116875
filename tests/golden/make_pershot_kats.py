"""Writes tests/golden/pershot_kats.json: known-answer cases of run()'s per-shot
path (mid-circuit measure / reset / if and stochastic noise) restated from the
reference's own test suite (dmvjs/ket, src/circuit.test.ts).

The reference cannot run in this environment (no Node), so each case carries
the circuit, the run() options and the assertions of the test it cites.

Case format: {"id", "cite", "n", "ops", "run": {"shots", "seed", "noise"},
"checks"} where ops are
  [gate, qubits, params]             a builder gate (as in reference_kats.json)
  ["creg", name, size]               creg()
  ["measure", q, creg, bit]          measure()
  ["reset", q, value]                reset(q, value)
  ["if", creg, value, [ops...]]      if()
noise is null, a device name, or {"p1", "p2", "pMeas"}; checks are
  ["creg", name, bit, x, digits]     cregs[name][bit] toBeCloseTo(x, digits)
  ["creg_near", name, bit, x, tol]   |cregs[name][bit] - x| <= tol
  ["creg_match", a, b, digits]       cregs[a][0] toBeCloseTo(cregs[b][0], digits)
  ["prob", bits, x, digits]          (probs[bits] ?? 0) toBeCloseTo(x, digits)
  ["prob_near", bits, x, tol]
  ["sum_gt", [bits...], x]           sum of probs over bits > x
  ["sum_lt", [bits...], x]
  ["keys_in", [bits...]]             every key of probs is listed
  ["keys_char", pos, ch]             every key has ch at position pos
  ["pos_close", pos, ch, x, digits]  sum of probs of keys with ch at pos, toBeCloseTo
  ["pos_near", pos, ch, x, tol]
  ["total", tol]                     |sum of probs - 1| < tol
  ["shots", k]
  ["like_clean", tol]                every probs value within tol of the noiseless run's
Run: python tests/golden/make_pershot_kats.py
"""
import json
import os

cases = []


def case(id_, cite, n, ops, shots, seed, checks, noise=None):
    cases.append({"id": id_, "cite": cite, "n": n, "ops": ops, "run": {"shots": shots, "seed": seed, "noise": noise},
                  "checks": checks})


X = lambda q: ["x", [q], []]  # noqa: E731
H = lambda q: ["h", [q], []]  # noqa: E731
Z = lambda q: ["z", [q], []]  # noqa: E731
CX = lambda c, t: ["cnot", [c, t], []]  # noqa: E731

# measure -- deterministic collapse (circuit.test.ts:1740-1760)
case("m_zero_creg", "circuit.test.ts:1741-1744", 1, [["measure", 0, "c", 0]], 100, 1, [["creg", "c", 0, 0.0, 10]])
case("m_one_creg", "circuit.test.ts:1746-1749", 1, [X(0), ["measure", 0, "c", 0]], 100, 1, [["creg", "c", 0, 1.0, 10]])
case("m_zero_stays", "circuit.test.ts:1751-1754", 1, [["measure", 0, "c", 0]], 100, 1, [["prob", "0", 1.0, 10]])
case("m_one_stays", "circuit.test.ts:1756-1759", 1, [X(0), ["measure", 0, "c", 0]], 100, 1, [["prob", "1", 1.0, 10]])
# measure -- superposition and collapse (:1762-1798)
case("m_plus_half", "circuit.test.ts:1763-1766", 1, [H(0), ["measure", 0, "c", 0]], 10000, 42,
     [["creg_near", "c", 0, 0.5, 0.05]])
case("m_collapse_real", "circuit.test.ts:1770-1774", 1, [H(0), ["measure", 0, "c", 0], H(0)], 10000, 42,
     [["prob_near", "0", 0.5, 0.05], ["prob_near", "1", 0.5, 0.05]])
case("m_remeasure", "circuit.test.ts:1776-1786", 1, [H(0), ["measure", 0, "c", 0], ["measure", 0, "c2", 0]], 10000, 42,
     [["creg_near", "c", 0, 0.5, 0.05], ["creg_near", "c2", 0, 0.5, 0.05], ["creg_match", "c", "c2", 1]])
case("m_bell", "circuit.test.ts:1788-1797", 2, [H(0), CX(0, 1), ["measure", 0, "c", 0]], 2000, 7,
     [["keys_in", ["00", "11"]]])
# measure -- multi-bit register (:1800-1817)
case("m_two_bits", "circuit.test.ts:1801-1811", 2, [X(0), ["creg", "c", 2], ["measure", 0, "c", 0], ["measure", 1, "c", 1]],
     100, 1, [["creg", "c", 0, 1.0, 10], ["creg", "c", 1, 0.0, 10]])
case("m_auto_creg", "circuit.test.ts:1813-1816", 1, [X(0), ["measure", 0, "auto", 0]], 100, 1,
     [["creg", "auto", 0, 1.0, 10]])
# reset (:1819-1861)
case("r_zero", "circuit.test.ts:1820-1823", 1, [["reset", 0, 0]], 100, 1, [["prob", "0", 1.0, 10]])
case("r_one", "circuit.test.ts:1825-1828", 1, [X(0), ["reset", 0, 0]], 100, 1, [["prob", "0", 1.0, 10]])
case("r_plus", "circuit.test.ts:1830-1833", 1, [H(0), ["reset", 0, 0]], 100, 1, [["prob", "0", 1.0, 10]])
case("r_bell", "circuit.test.ts:1835-1840", 2, [H(0), CX(0, 1), ["reset", 0, 0]], 100, 1, [["keys_char", 0, "0"]])
case("r_to_one", "circuit.test.ts:1842-1845", 1, [["reset", 0, 1]], 100, 1, [["prob", "1", 1.0, 10]])
case("r_zero_to_one", "circuit.test.ts:1847-1850", 1, [["reset", 0, 1]], 100, 1, [["prob", "1", 1.0, 10]])
case("r_plus_to_one", "circuit.test.ts:1852-1855", 1, [H(0), ["reset", 0, 1]], 100, 1, [["prob", "1", 1.0, 10]])
case("r_value0", "circuit.test.ts:1857-1861", 1, [X(0), ["reset", 0, 0]], 100, 1, [["prob", "0", 1.0, 10]])
# if (:1864-1966)
case("if_zero_fires", "circuit.test.ts:1865-1869", 1, [["measure", 0, "c", 0], ["if", "c", 0, [X(0)]]], 100, 1,
     [["prob", "1", 1.0, 10]])
case("if_one_fires", "circuit.test.ts:1871-1875", 1, [X(0), ["measure", 0, "c", 0], ["if", "c", 1, [X(0)]]], 100, 1,
     [["prob", "0", 1.0, 10]])
case("if_one_skips", "circuit.test.ts:1877-1881", 1, [X(0), ["measure", 0, "c", 0], ["if", "c", 0, [X(0)]]], 100, 1,
     [["prob", "1", 1.0, 10]])
case("if_corrects", "circuit.test.ts:1883-1887", 1, [H(0), ["measure", 0, "c", 0], ["if", "c", 1, [X(0)]]], 1000, 42,
     [["prob", "0", 1.0, 5]])
case("if_value2", "circuit.test.ts:1889-1898", 2,
     [X(1), ["creg", "c", 2], ["measure", 0, "c", 0], ["measure", 1, "c", 1], ["if", "c", 2, [X(0)]]], 100, 1,
     [["prob", "11", 1.0, 10]])
case("if_value1_skips", "circuit.test.ts:1900-1909", 2,
     [X(1), ["creg", "c", 2], ["measure", 0, "c", 0], ["measure", 1, "c", 1], ["if", "c", 1, [X(0)]]], 100, 1,
     [["prob", "01", 1.0, 10]])
case("if_value3", "circuit.test.ts:1911-1920", 3,
     [X(0), X(1), ["creg", "c", 2], ["measure", 0, "c", 0], ["measure", 1, "c", 1], ["if", "c", 3, [X(2)]]], 100, 1,
     [["prob", "111", 1.0, 10]])


def teleport(prep):
    return prep + [H(1), CX(1, 2), CX(0, 1), H(0), ["measure", 0, "c0", 0], ["measure", 1, "c1", 0],
                   ["if", "c1", 1, [X(2)]], ["if", "c0", 1, [Z(2)]]]


case("tele_zero", "circuit.test.ts:1931-1950", 3, teleport([]), 1000, 1, [["pos_close", 2, "0", 1.0, 5]])
case("tele_one", "circuit.test.ts:1931-1957", 3, teleport([X(0)]), 1000, 1, [["pos_close", 2, "1", 1.0, 5]])
case("tele_plus", "circuit.test.ts:1931-1965", 3, teleport([H(0)]), 1000, 1,
     [["pos_near", 2, "0", 0.5, 0.05], ["pos_near", 2, "1", 0.5, 0.05]])
# measure + reset (:1968-1980)
case("m_then_reset", "circuit.test.ts:1968-1973", 1, [X(0), ["measure", 0, "c", 0], ["reset", 0, 0]], 100, 1,
     [["creg", "c", 0, 1.0, 10], ["prob", "0", 1.0, 10]])
case("reset_reuse", "circuit.test.ts:1975-1979", 1, [X(0), ["measure", 0, "c", 0], ["reset", 0, 0], X(0)], 100, 1,
     [["prob", "1", 1.0, 10]])
# noise: depolarizing, single-qubit (:2395-2420)
case("n_clean_x", "circuit.test.ts:2396-2399", 1, [X(0)], 200, 1, [["prob", "1", 1.0, 10]])
case("n_p1_high", "circuit.test.ts:2401-2407", 1, [X(0)], 4000, 1, [["sum_gt", ["0"], 0.1], ["sum_lt", ["1"], 0.9]],
     noise={"p1": 0.5})
case("n_p1_small", "circuit.test.ts:2409-2413", 1, [X(0)], 10000, 2, [["sum_gt", ["1"], 0.99]], noise={"p1": 0.001})
case("n_p1_zero", "circuit.test.ts:2415-2419", 1, [H(0)], 4000, 7, [["like_clean", 0.05]], noise={"p1": 0})
# two-qubit (:2422-2436)
case("n_p2_high", "circuit.test.ts:2423-2430", 2, [H(0), CX(0, 1)], 2000, 1, [["sum_gt", ["01", "10"], 0.05]],
     noise={"p2": 0.5})
case("n_p2_small", "circuit.test.ts:2432-2435", 2, [H(0), CX(0, 1)], 10000, 3, [["sum_gt", ["00", "11"], 0.95]],
     noise={"p2": 0.005})
# SPAM (:2438-2456)
case("n_pm_one", "circuit.test.ts:2439-2444", 1, [X(0)], 200, 1, [["prob", "0", 1.0, 5]], noise={"pMeas": 1})
case("n_pm_half", "circuit.test.ts:2446-2451", 1, [X(0)], 4000, 4,
     [["prob_near", "0", 0.5, 0.05], ["prob_near", "1", 0.5, 0.05]], noise={"pMeas": 0.5})
case("n_pm_small", "circuit.test.ts:2453-2456", 1, [X(0)], 10000, 5, [["sum_gt", ["1"], 0.99]], noise={"pMeas": 0.004})
# named device profiles (:2458-2482)
case("n_aria", "circuit.test.ts:2459-2463", 2, [H(0), CX(0, 1)], 1000, 1, [["total", 0.001]], noise="aria-1")
case("n_forte", "circuit.test.ts:2465-2468", 1, [H(0)], 1000, 2, [["shots", 1000]], noise="forte-1")
case("n_harmony", "circuit.test.ts:2470-2473", 1, [X(0)], 500, 3, [["shots", 500]], noise="harmony")
case("n_aria_bell", "circuit.test.ts:2475-2478", 2, [H(0), CX(0, 1)], 5000, 10, [["sum_gt", ["00", "11"], 0.97]],
     noise="aria-1")
# custom NoiseParams (:2485-2498)
case("n_custom", "circuit.test.ts:2486-2491", 2, [H(0), CX(0, 1)], 2000, 99,
     [["shots", 2000], ["sum_gt", ["00", "11"], 0.97]], noise={"p1": 0.0003, "p2": 0.005, "pMeas": 0.004})
case("n_only_p1", "circuit.test.ts:2493-2496", 1, [H(0)], 2000, 1, [["prob_near", "0", 0.5, 0.06]],
     noise={"p1": 0.001})

if __name__ == "__main__":
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pershot_kats.json")
    with open(out, "w") as f:
        json.dump({"source": "dmvjs/ket src/circuit.test.ts (restated)", "cases": cases}, f, indent=1)
    print(out, len(cases))
