// json_loader.cpp -- ket's circuit JSON (schema "ket": 1) for hosts without
// Node: Circuit.fromJSON (circuit.ts:3794-3806) and opsFromJSON (:532-580)
// lowered straight to the C ABI's op list.
//
// The loader parses the text, rebuilds every gate matrix from its name and
// parameters as gate2x2FromMeta / gate4x4FromMeta / ctrlGate2x2FromMeta do
// (:467-529, matrices of gates.ts:11-208), inlines named sub-circuits with
// their qubits remapped (flattenOps, :113-133) and packs measure / reset / if
// in ket_run_shots' encoding, with the registers of "cregs" numbered
// consecutively in the file's order.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "ctx.h"

using namespace ket;

namespace {

// ---------------------------------------------------------------- JSON values
struct JV {
  enum T { NUL, BOOL, NUM, STR, ARR, OBJ } t = NUL;
  bool b = false;
  double n = 0;
  std::string s;
  std::vector<JV> a;
  std::vector<std::pair<std::string, JV>> o;
  const JV* get(const char* k) const {
    for (const auto& kv : o)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
};

struct Parser {
  const char* p;
  const char* e;
  std::string err;
  int depth = 0;

  void ws() {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
  }
  bool fail(const std::string& m) {
    if (err.empty()) err = m;
    return false;
  }
  static void utf8(std::string& out, uint32_t c) {
    if (c < 0x80) out += (char)c;
    else if (c < 0x800) { out += (char)(0xC0 | (c >> 6)); out += (char)(0x80 | (c & 0x3F)); }
    else if (c < 0x10000) {
      out += (char)(0xE0 | (c >> 12)); out += (char)(0x80 | ((c >> 6) & 0x3F)); out += (char)(0x80 | (c & 0x3F));
    } else {
      out += (char)(0xF0 | (c >> 18)); out += (char)(0x80 | ((c >> 12) & 0x3F));
      out += (char)(0x80 | ((c >> 6) & 0x3F)); out += (char)(0x80 | (c & 0x3F));
    }
  }
  bool hex4(uint32_t& v) {
    if (e - p < 4) return fail("JSON: short \\u escape");
    v = 0;
    for (int i = 0; i < 4; i++) {
      const char ch = *p++;
      v <<= 4;
      if (ch >= '0' && ch <= '9') v |= ch - '0';
      else if (ch >= 'a' && ch <= 'f') v |= ch - 'a' + 10;
      else if (ch >= 'A' && ch <= 'F') v |= ch - 'A' + 10;
      else return fail("JSON: bad \\u escape");
    }
    return true;
  }
  bool str(std::string& out) {
    p++;  // opening quote
    while (p < e && *p != '"') {
      const unsigned char ch = (unsigned char)*p;
      if (ch < 0x20) return fail("JSON: control character in string");
      if (ch != '\\') { out += (char)ch; p++; continue; }
      if (++p >= e) return fail("JSON: unterminated escape");
      const char x = *p++;
      switch (x) {
        case '"': out += '"'; break;
        case '\\': out += '\\'; break;
        case '/': out += '/'; break;
        case 'b': out += '\b'; break;
        case 'f': out += '\f'; break;
        case 'n': out += '\n'; break;
        case 'r': out += '\r'; break;
        case 't': out += '\t'; break;
        case 'u': {
          uint32_t c;
          if (!hex4(c)) return false;
          if (c >= 0xD800 && c < 0xDC00 && e - p >= 6 && p[0] == '\\' && p[1] == 'u') {
            p += 2;
            uint32_t lo;
            if (!hex4(lo)) return false;
            if (lo >= 0xDC00 && lo < 0xE000) c = 0x10000 + ((c - 0xD800) << 10) + (lo - 0xDC00);
            else { utf8(out, c); c = lo; }
          }
          utf8(out, c);
          break;
        }
        default: return fail("JSON: bad escape");
      }
    }
    if (p >= e) return fail("JSON: unterminated string");
    p++;
    return true;
  }
  bool num(double& v) {
    const char* s = p;
    if (p < e && *p == '-') p++;
    if (p >= e || !(*p >= '0' && *p <= '9')) return fail("JSON: bad number");
    if (*p == '0') p++;
    else while (p < e && *p >= '0' && *p <= '9') p++;
    if (p < e && *p == '.') {
      p++;
      if (p >= e || !(*p >= '0' && *p <= '9')) return fail("JSON: bad number");
      while (p < e && *p >= '0' && *p <= '9') p++;
    }
    if (p < e && (*p == 'e' || *p == 'E')) {
      p++;
      if (p < e && (*p == '+' || *p == '-')) p++;
      if (p >= e || !(*p >= '0' && *p <= '9')) return fail("JSON: bad number");
      while (p < e && *p >= '0' && *p <= '9') p++;
    }
    const std::string t(s, p);
    v = strtod(t.c_str(), nullptr);
    return true;
  }
  bool lit(const char* w) {
    const size_t k = strlen(w);
    if ((size_t)(e - p) < k || strncmp(p, w, k) != 0) return fail("JSON: bad literal");
    p += k;
    return true;
  }
  bool value(JV& v) {
    if (++depth > 256) return fail("JSON: nested too deeply");
    ws();
    if (p >= e) return fail("JSON: unexpected end");
    bool ok = true;
    switch (*p) {
      case '{': {
        v.t = JV::OBJ;
        p++;
        ws();
        if (p < e && *p == '}') { p++; break; }
        while (true) {
          ws();
          if (p >= e || *p != '"') { ok = fail("JSON: expected a key"); break; }
          std::string k;
          if (!str(k)) { ok = false; break; }
          ws();
          if (p >= e || *p != ':') { ok = fail("JSON: expected ':'"); break; }
          p++;
          JV x;
          if (!value(x)) { ok = false; break; }
          // a repeated key keeps its first position and its last value, as JSON.parse does
          bool found = false;
          for (auto& kv : v.o)
            if (kv.first == k) { kv.second = std::move(x); found = true; break; }
          if (!found) v.o.emplace_back(std::move(k), std::move(x));
          ws();
          if (p < e && *p == ',') { p++; continue; }
          if (p < e && *p == '}') { p++; break; }
          ok = fail("JSON: expected ',' or '}'");
          break;
        }
        break;
      }
      case '[': {
        v.t = JV::ARR;
        p++;
        ws();
        if (p < e && *p == ']') { p++; break; }
        while (true) {
          JV x;
          if (!value(x)) { ok = false; break; }
          v.a.push_back(std::move(x));
          ws();
          if (p < e && *p == ',') { p++; continue; }
          if (p < e && *p == ']') { p++; break; }
          ok = fail("JSON: expected ',' or ']'");
          break;
        }
        break;
      }
      case '"': v.t = JV::STR; ok = str(v.s); break;
      case 't': v.t = JV::BOOL; v.b = true; ok = lit("true"); break;
      case 'f': v.t = JV::BOOL; v.b = false; ok = lit("false"); break;
      case 'n': v.t = JV::NUL; ok = lit("null"); break;
      default: v.t = JV::NUM; ok = num(v.n); break;
    }
    depth--;
    return ok;
  }
};

// ---------------------------------------------------------------- gate matrices (gates.ts:11-208)
typedef std::vector<std::pair<double, double>> M;
const double SQ2 = 1 / std::sqrt(2.0);

M m2(double a, double b, double c, double d, double e, double f, double g, double h) {
  return {{a, b}, {c, d}, {e, f}, {g, h}};
}
M gRx(double t) { const double c = std::cos(t / 2), s = std::sin(t / 2); return m2(c, 0, 0, -s, 0, -s, c, 0); }
M gRy(double t) { const double c = std::cos(t / 2), s = std::sin(t / 2); return m2(c, 0, -s, 0, s, 0, c, 0); }
M gRz(double t) { const double c = std::cos(t / 2), s = std::sin(t / 2); return m2(c, -s, 0, 0, 0, 0, c, s); }
M gU3(double t, double p, double l) {
  const double c = std::cos(t / 2), s = std::sin(t / 2);
  return m2(c, 0, -s * std::cos(l), -s * std::sin(l), s * std::cos(p), s * std::sin(p), c * std::cos(p + l),
            c * std::sin(p + l));
}
M gU1(double l) { return m2(1, 0, 0, 0, 0, 0, std::cos(l), std::sin(l)); }
M gGpi(double p) { const double c = std::cos(p), s = std::sin(p); return m2(0, 0, c, -s, c, s, 0, 0); }
M gGpi2(double p) {
  const double c = std::cos(p), s = std::sin(p);
  return m2(SQ2, 0, -SQ2 * s, -SQ2 * c, SQ2 * s, -SQ2 * c, SQ2, 0);
}
M four(const std::pair<double, double> (&v)[16]) { return M(v, v + 16); }
M gXx(double t) {
  const double c = std::cos(t / 2), n = -std::sin(t / 2);
  const std::pair<double, double> v[16] = {{c, 0}, {0, 0}, {0, 0}, {0, n}, {0, 0}, {c, 0}, {0, n}, {0, 0},
                                           {0, 0}, {0, n}, {c, 0}, {0, 0}, {0, n}, {0, 0}, {0, 0}, {c, 0}};
  return four(v);
}
M gYy(double t) {
  const double c = std::cos(t / 2), n = -std::sin(t / 2), p = std::sin(t / 2);
  const std::pair<double, double> v[16] = {{c, 0}, {0, 0}, {0, 0}, {0, p}, {0, 0}, {c, 0}, {0, n}, {0, 0},
                                           {0, 0}, {0, n}, {c, 0}, {0, 0}, {0, p}, {0, 0}, {0, 0}, {c, 0}};
  return four(v);
}
M gZz(double t) {
  const double c = std::cos(t / 2), s = std::sin(t / 2);
  const std::pair<double, double> v[16] = {{c, -s}, {0, 0}, {0, 0}, {0, 0}, {0, 0}, {c, s}, {0, 0}, {0, 0},
                                           {0, 0}, {0, 0}, {c, s}, {0, 0}, {0, 0}, {0, 0}, {0, 0}, {c, -s}};
  return four(v);
}
M gXy(double t) {
  const double c = std::cos(t / 2), s = std::sin(t / 2);
  const std::pair<double, double> v[16] = {{1, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}, {c, 0}, {0, s}, {0, 0},
                                           {0, 0}, {0, s}, {c, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}, {1, 0}};
  return four(v);
}
M gMs(double p0, double p1) {
  const double sp = std::sin(p0 + p1), cp = std::cos(p0 + p1), sd = std::sin(p0 - p1), cd = std::cos(p0 - p1);
  const std::pair<double, double> v[16] = {
      {SQ2, 0}, {0, 0}, {0, 0}, {-sp * SQ2, -cp * SQ2}, {0, 0}, {SQ2, 0}, {-sd * SQ2, -cd * SQ2}, {0, 0},
      {0, 0}, {sd * SQ2, -cd * SQ2}, {SQ2, 0}, {0, 0}, {sp * SQ2, -cp * SQ2}, {0, 0}, {0, 0}, {SQ2, 0}};
  return four(v);
}

// the fixed single-qubit matrices (gates.ts:13-24)
bool fixed1(const std::string& n, M& m) {
  if (n == "id") m = m2(1, 0, 0, 0, 0, 0, 1, 0);
  else if (n == "h") m = m2(SQ2, 0, SQ2, 0, SQ2, 0, -SQ2, 0);
  else if (n == "x") m = m2(0, 0, 1, 0, 1, 0, 0, 0);
  else if (n == "y") m = m2(0, 0, 0, -1, 0, 1, 0, 0);
  else if (n == "z") m = m2(1, 0, 0, 0, 0, 0, -1, 0);
  else if (n == "s") m = m2(1, 0, 0, 0, 0, 0, 0, 1);
  else if (n == "si" || n == "sdg") m = m2(1, 0, 0, 0, 0, 0, 0, -1);
  else if (n == "t") m = m2(1, 0, 0, 0, 0, 0, SQ2, SQ2);
  else if (n == "ti" || n == "tdg") m = m2(1, 0, 0, 0, 0, 0, SQ2, -SQ2);
  else if (n == "v" || n == "srn" || n == "sx") m = m2(.5, .5, .5, -.5, .5, -.5, .5, .5);
  else if (n == "vi" || n == "srndg" || n == "sxdg") m = m2(.5, -.5, .5, .5, .5, .5, .5, -.5);
  else if (n == "r2") m = gRz(M_PI / 2);
  else if (n == "r4") m = gRz(M_PI / 4);
  else if (n == "r8") m = gRz(M_PI / 8);
  else return false;
  return true;
}

double par(const std::vector<double>& p, size_t i) { return i < p.size() ? p[i] : std::nan(""); }

// gate2x2FromMeta (circuit.ts:467-484)
bool single_from_meta(const std::string& n, const std::vector<double>& p, M& m) {
  if (fixed1(n, m)) return true;
  if (n == "rx") m = gRx(par(p, 0));
  else if (n == "ry") m = gRy(par(p, 0));
  else if (n == "rz" || n == "vz") m = gRz(par(p, 0));
  else if (n == "u1" || n == "p") m = gU1(par(p, 0));
  else if (n == "u2") m = gU3(M_PI / 2, par(p, 0), par(p, 1));
  else if (n == "u3") m = gU3(par(p, 0), par(p, 1), par(p, 2));
  else if (n == "gpi") m = gGpi(par(p, 0));
  else if (n == "gpi2") m = gGpi2(par(p, 0));
  else return false;
  return true;
}
// gate4x4FromMeta (:487-499)
bool two_from_meta(const std::string& n, const std::vector<double>& p, M& m) {
  if (n == "xx") m = gXx(par(p, 0));
  else if (n == "yy") m = gYy(par(p, 0));
  else if (n == "zz") m = gZz(par(p, 0));
  else if (n == "xy") m = gXy(par(p, 0));
  else if (n == "iswap") m = gXy(M_PI);
  else if (n == "srswap") m = gXy(M_PI / 2);
  else if (n == "ms") m = gMs(par(p, 0), par(p, 1));
  else return false;
  return true;
}
// ctrlGate2x2FromMeta (:502-515)
bool ctrl_from_meta(const std::string& n, const std::vector<double>& p, M& m) {
  if (n == "cx") m = m2(0, 0, 1, 0, 1, 0, 0, 0);
  else if (n == "cy") return fixed1("y", m);
  else if (n == "cz") return fixed1("z", m);
  else if (n == "ch") return fixed1("h", m);
  else if (n == "crx") m = gRx(par(p, 0));
  else if (n == "cry") m = gRy(par(p, 0));
  else if (n == "crz") m = gRz(par(p, 0));
  else if (n == "cu1") m = gU1(par(p, 0));
  else if (n == "cu2") m = gU3(M_PI / 2, par(p, 0), par(p, 1));
  else if (n == "cu3") m = gU3(par(p, 0), par(p, 1), par(p, 2));
  else if (n == "cs") return fixed1("s", m);
  else if (n == "ct") return fixed1("t", m);
  else if (n == "csdg") return fixed1("si", m);
  else if (n == "ctdg") return fixed1("ti", m);
  else if (n == "cr2") return fixed1("r2", m);
  else if (n == "cr4") return fixed1("r4", m);
  else if (n == "cr8") return fixed1("r8", m);
  else if (n == "csrn") return fixed1("v", m);
  else return false;
  return true;
}

}  // namespace

struct ket_program {
  int nqubits = 0;
  std::vector<ket_op> ops;
  std::vector<double> mats;  // interleaved (re, im)
  std::vector<std::pair<std::string, int>> cregs;
  std::vector<int> first;    // first classical bit of each register
  int ncbits = 0;
  bool classical = false;
};

namespace {

struct Lower {
  ket_program* P;
  std::string err;
  int code = KET_OK;
  std::vector<std::string> unbound;

  bool bad(int c, const std::string& m) {
    if (code == KET_OK) { code = c; err = m; }
    return false;
  }
  bool num(const JV* v, double& out) {
    if (!v || v->t != JV::NUM) return false;
    out = v->n;
    return true;
  }
  bool qubit(const JV& o, const char* k, const std::vector<int>& qmap, int& q) {
    double d;
    if (!num(o.get(k), d) || d != std::floor(d) || std::fabs(d) > 1e9)
      return bad(KET_ERR_TYPE, std::string("fromJSON: op field '") + k + "' must be an integer");
    const int i = (int)d;
    if (qmap.empty()) { q = i; return true; }
    if (i < 0 || i >= (int)qmap.size()) return bad(KET_ERR_RANGE, "fromJSON: sub-circuit qubit out of range");
    q = qmap[i];
    return true;
  }
  bool params(const JV& o, std::string& name, std::vector<double>& ps) {
    const JV* meta = o.get("meta");
    if (!meta || meta->t != JV::OBJ) return bad(KET_ERR_TYPE, "fromJSON: gate op without meta");
    const JV* n = meta->get("name");
    if (!n || n->t != JV::STR) return bad(KET_ERR_TYPE, "fromJSON: meta without a name");
    name = n->s;
    const JV* pa = meta->get("params");
    if (pa && pa->t == JV::ARR)
      for (const JV& x : pa->a) ps.push_back(x.t == JV::NUM ? x.n : std::nan(""));
    return true;
  }
  void emit(int kind, std::initializer_list<int> qs, const M* m) {
    ket_op o;
    memset(&o, 0, sizeof(o));
    o.kind = kind;
    o.nq = (int)qs.size();
    int j = 0;
    for (int q : qs) o.q[j++] = q;
    o.mat = -1;
    if (m) {
      o.mat = (int64_t)(P->mats.size() / 2);
      for (const auto& z : *m) { P->mats.push_back(z.first); P->mats.push_back(z.second); }
    }
    P->ops.push_back(o);
  }
  int reg_first(const std::string& name, int& size) {
    for (size_t i = 0; i < P->cregs.size(); i++)
      if (P->cregs[i].first == name) { size = P->cregs[i].second; return P->first[i]; }
    size = 0;
    return -1;
  }
  // opsFromJSON + flattenOps over one op list; qmap maps sub-circuit qubits
  bool ops(const JV& list, const std::vector<int>& qmap, int depth) {
    if (list.t != JV::ARR) return bad(KET_ERR_TYPE, "fromJSON: ops must be an array");
    if (depth > 64) return bad(KET_ERR_TYPE, "fromJSON: sub-circuits nested too deeply");
    for (const JV& o : list.a) {
      if (o.t != JV::OBJ) return bad(KET_ERR_TYPE, "fromJSON: op must be an object");
      const JV* k = o.get("kind");
      const std::string kind = k && k->t == JV::STR ? k->s : std::string("?");
      int a, b, c;
      std::string name;
      std::vector<double> ps;
      M m;
      if (kind == "single") {
        if (!qubit(o, "q", qmap, a) || !params(o, name, ps)) return false;
        if (!single_from_meta(name, ps, m)) return bad(KET_ERR_TYPE, "fromJSON: unknown single-qubit gate '" + name + "'");
        emit(KET_OP_SINGLE, {a}, &m);
      } else if (kind == "cnot") {
        if (!qubit(o, "control", qmap, a) || !qubit(o, "target", qmap, b)) return false;
        emit(KET_OP_CNOT, {a, b}, nullptr);
      } else if (kind == "swap") {
        if (!qubit(o, "a", qmap, a) || !qubit(o, "b", qmap, b)) return false;
        emit(KET_OP_SWAP, {a, b}, nullptr);
      } else if (kind == "two") {
        if (!qubit(o, "a", qmap, a) || !qubit(o, "b", qmap, b) || !params(o, name, ps)) return false;
        if (!two_from_meta(name, ps, m)) return bad(KET_ERR_TYPE, "fromJSON: unknown two-qubit gate '" + name + "'");
        emit(KET_OP_TWO, {a, b}, &m);
      } else if (kind == "controlled") {
        if (!qubit(o, "control", qmap, a) || !qubit(o, "target", qmap, b) || !params(o, name, ps)) return false;
        if (!ctrl_from_meta(name, ps, m)) return bad(KET_ERR_TYPE, "fromJSON: unknown controlled gate '" + name + "'");
        emit(KET_OP_CONTROLLED, {a, b}, &m);
      } else if (kind == "toffoli") {
        if (!qubit(o, "c1", qmap, a) || !qubit(o, "c2", qmap, b) || !qubit(o, "target", qmap, c)) return false;
        emit(KET_OP_TOFFOLI, {a, b, c}, nullptr);
      } else if (kind == "cswap" || kind == "csrswap") {
        if (!qubit(o, "control", qmap, a) || !qubit(o, "a", qmap, b) || !qubit(o, "b", qmap, c)) return false;
        emit(kind == "cswap" ? KET_OP_CSWAP : KET_OP_CSRSWAP, {a, b, c}, nullptr);
      } else if (kind == "barrier") {
        // no effect on the state: kept with its qubits (its first one only past 10)
        const JV* qs = o.get("qubits");
        if (!qs || qs->t != JV::ARR) return bad(KET_ERR_TYPE, "fromJSON: barrier without qubits");
        ket_op x;
        memset(&x, 0, sizeof(x));
        x.kind = KET_OP_BARRIER;
        x.mat = -1;
        const size_t k = qs->a.size() > KET_MAX_OP_QUBITS ? 1 : qs->a.size();
        for (size_t i = 0; i < k; i++) {
          if (qs->a[i].t != JV::NUM) return bad(KET_ERR_TYPE, "fromJSON: barrier qubit");
          const int q = (int)qs->a[i].n;
          if (!qmap.empty() && (q < 0 || q >= (int)qmap.size())) return bad(KET_ERR_RANGE, "fromJSON: sub-circuit qubit out of range");
          x.q[x.nq++] = qmap.empty() ? q : qmap[q];
        }
        P->ops.push_back(x);
      } else if (kind == "unitary") {
        const JV* qs = o.get("qubits");
        const JV* mat = o.get("matrix");
        if (!qs || qs->t != JV::ARR || !mat || mat->t != JV::ARR) return bad(KET_ERR_TYPE, "fromJSON: unitary fields");
        const size_t k = qs->a.size();
        if (k == 0 || k > KET_MAX_OP_QUBITS) return bad(KET_ERR_TYPE, "unitary: 1 to 10 qubits");
        const size_t d = size_t(1) << k;
        if (mat->a.size() != d) return bad(KET_ERR_TYPE, "unitary: matrix shape");
        ket_op x;
        memset(&x, 0, sizeof(x));
        x.kind = KET_OP_UNITARY;
        x.nq = (int)k;
        for (size_t i = 0; i < k; i++) {
          if (qs->a[i].t != JV::NUM) return bad(KET_ERR_TYPE, "fromJSON: unitary qubit");
          const int q = (int)qs->a[i].n;
          if (!qmap.empty() && (q < 0 || q >= (int)qmap.size())) return bad(KET_ERR_RANGE, "fromJSON: sub-circuit qubit out of range");
          x.q[i] = qmap.empty() ? q : qmap[q];
        }
        x.mat = (int64_t)(P->mats.size() / 2);
        for (const JV& row : mat->a) {
          if (row.t != JV::ARR || row.a.size() != d) return bad(KET_ERR_TYPE, "unitary: matrix shape");
          for (const JV& z : row.a) {
            if (z.t != JV::ARR || z.a.size() != 2 || z.a[0].t != JV::NUM || z.a[1].t != JV::NUM)
              return bad(KET_ERR_TYPE, "unitary: entries must be [re, im]");
            P->mats.push_back(z.a[0].n);
            P->mats.push_back(z.a[1].n);
          }
        }
        P->ops.push_back(x);
      } else if (kind == "measure") {
        // remapOp leaves measure / reset / if as they are (circuit.ts:102-104)
        if (!qubit(o, "q", {}, a)) return false;
        const JV* cr = o.get("creg");
        double bit;
        if (!cr || cr->t != JV::STR || !num(o.get("bit"), bit)) return bad(KET_ERR_TYPE, "fromJSON: measure fields");
        int size;
        const int f = reg_first(cr->s, size);
        const int cb = f >= 0 && bit >= 0 && bit < size && bit == std::floor(bit) ? f + (int)bit : -1;
        emit(KET_OP_MEASURE, {a, cb}, nullptr);
        P->classical = true;
      } else if (kind == "reset") {
        if (!qubit(o, "q", {}, a)) return false;
        emit(KET_OP_RESET, {a}, nullptr);
        P->classical = true;
      } else if (kind == "if") {
        const JV* cr = o.get("creg");
        double value;
        const JV* body = o.get("ops");
        if (!cr || cr->t != JV::STR || !num(o.get("value"), value) || !body)
          return bad(KET_ERR_TYPE, "fromJSON: if fields");
        int size;
        int f = reg_first(cr->s, size);
        if (f < 0) { f = 0; size = 0; }
        if (size > 31) return bad(KET_ERR_UNSUPPORTED, "if() on a register of more than 31 bits");
        // a value that no register of <= 31 bits can hold never matches
        const int v = value == std::floor(value) && value >= -2147483648.0 && value < 2147483648.0 ? (int)value : -1;
        const size_t at = P->ops.size();
        emit(KET_OP_IF, {f, size, v, 0}, nullptr);
        if (!ops(*body, {}, depth + 1)) return false;
        P->ops[at].q[3] = (int)(P->ops.size() - at - 1);
        P->classical = true;
      } else if (kind == "subcircuit") {
        const JV* qs = o.get("qubits");
        const JV* def = o.get("def");
        if (!qs || qs->t != JV::ARR || !def) return bad(KET_ERR_TYPE, "fromJSON: subcircuit fields");
        std::vector<int> sub;
        for (const JV& x : qs->a) {
          if (x.t != JV::NUM) return bad(KET_ERR_TYPE, "fromJSON: subcircuit qubit");
          const int q = (int)x.n;
          if (!qmap.empty() && (q < 0 || q >= (int)qmap.size())) return bad(KET_ERR_RANGE, "fromJSON: sub-circuit qubit out of range");
          sub.push_back(qmap.empty() ? q : qmap[q]);
        }
        if (!ops(*def, sub, depth + 1)) return false;
      } else if (kind == "parametric") {
        // flattenOps refuses unbound parameters (circuit.ts:117-121)
        const JV* pa = o.get("params");
        if (pa && pa->t == JV::ARR)
          for (const JV& x : pa->a)
            if (x.t == JV::STR) unbound.push_back(x.s);
        if (unbound.empty()) unbound.push_back("?");
      } else {
        return bad(KET_ERR_TYPE, "fromJSON: unknown op kind '" + kind + "'");
      }
    }
    return true;
  }
};

}  // namespace

extern "C" {

int ket_program_from_json(const char* text, size_t len, ket_program** out) {
  if (!text || !out) return fail(KET_ERR_TYPE, "null argument");
  *out = nullptr;
  Parser ps{text, text + len, "", 0};
  JV root;
  if (!ps.value(root)) return fail(KET_ERR_TYPE, ps.err);
  ps.ws();
  if (ps.p != ps.e) return fail(KET_ERR_TYPE, "JSON: trailing characters");
  if (root.t != JV::OBJ) return fail(KET_ERR_TYPE, "fromJSON: expected an object");
  const JV* ver = root.get("ket");
  if (!ver || ver->t != JV::NUM || ver->n != 1)
    return fail(KET_ERR_TYPE, "fromJSON: unsupported schema version " +
                                  (ver && ver->t == JV::NUM ? std::to_string((long long)ver->n) : std::string("?")));
  const JV* nq = root.get("qubits");
  if (!nq || nq->t != JV::NUM || nq->n != std::floor(nq->n) || nq->n < 0 || nq->n > KET_MAX_QUBITS)
    return fail(KET_ERR_TYPE, "fromJSON: qubits must be an integer in [0, 40]");
  ket_program* P = new ket_program();
  P->nqubits = (int)nq->n;
  const JV* cr = root.get("cregs");
  if (cr && cr->t == JV::OBJ)
    for (const auto& kv : cr->o) {
      const int size = kv.second.t == JV::NUM && kv.second.n >= 0 && kv.second.n < 1e6 ? (int)kv.second.n : 0;
      P->cregs.emplace_back(kv.first, size);
      P->first.push_back(P->ncbits);
      P->ncbits += size;
    }
  const JV* ops = root.get("ops");
  Lower L{P, "", KET_OK, {}};
  if (!ops || !L.ops(*ops, {}, 0)) {
    delete P;
    return fail(L.code == KET_OK ? KET_ERR_TYPE : L.code, L.err.empty() ? "fromJSON: ops missing" : L.err);
  }
  if (!L.unbound.empty()) {
    std::string names;
    for (size_t i = 0; i < L.unbound.size(); i++) names += (i ? ", " : "") + L.unbound[i];
    delete P;
    return fail(KET_ERR_TYPE, "Circuit has unbound parameters: [" + names + "]. Call bind() first.");
  }
  *out = P;
  return KET_OK;
}

int ket_program_free(ket_program* p) {
  delete p;
  return KET_OK;
}

int ket_program_info(const ket_program* p, int* nqubits, size_t* nops, size_t* nmat, int* ncbits, int* nregs,
                     int* classical) {
  if (!p) return fail(KET_ERR_TYPE, "null program");
  if (nqubits) *nqubits = p->nqubits;
  if (nops) *nops = p->ops.size();
  if (nmat) *nmat = p->mats.size() / 2;
  if (ncbits) *ncbits = p->ncbits;
  if (nregs) *nregs = (int)p->cregs.size();
  if (classical) *classical = p->classical ? 1 : 0;
  return KET_OK;
}

int ket_program_ops(const ket_program* p, ket_op* ops, size_t ops_cap, double* mats, size_t mat_cap) {
  if (!p) return fail(KET_ERR_TYPE, "null program");
  if (ops_cap < p->ops.size() || mat_cap < p->mats.size() / 2) return fail(KET_ERR_TYPE, "output buffers too small");
  if (!p->ops.empty()) {
    if (!ops) return fail(KET_ERR_TYPE, "null op buffer");
    memcpy(ops, p->ops.data(), sizeof(ket_op) * p->ops.size());
  }
  if (!p->mats.empty()) {
    if (!mats) return fail(KET_ERR_TYPE, "null matrix buffer");
    memcpy(mats, p->mats.data(), sizeof(double) * p->mats.size());
  }
  return KET_OK;
}

int ket_program_creg(const ket_program* p, int i, char* name, size_t cap, int* first, int* size) {
  if (!p) return fail(KET_ERR_TYPE, "null program");
  if (i < 0 || i >= (int)p->cregs.size()) return fail(KET_ERR_RANGE, "register index out of range");
  if (name && cap) {
    const std::string& s = p->cregs[i].first;
    const size_t k = s.size() < cap - 1 ? s.size() : cap - 1;
    memcpy(name, s.data(), k);
    name[k] = 0;
  }
  if (first) *first = p->first[i];
  if (size) *size = p->cregs[i].second;
  return KET_OK;
}

}  // extern "C"
