// Native decoder for the circuit JSON the reference hands its core.
//
// The reference serialises a circuit with `circuit.model_dump_json()` and
// serde decodes it into `Circuit` / `Register` / `Instruction`
// (src/types.rs:8-135; the boundary call is statevector/simulator.rs:327-329).
// This file decodes that text straight into the dq_inst / dq_cond records of
// the C ABI, with the rules of the package's Python decoder (circuit.py:
// variant tags, required fields, ignored unknown keys, usize / f64 typing,
// num_qubits = max(base + size)) and its encoder (flattened condition
// chains, generic gate names matched lower-cased, qubit and classical-bit
// limits).
//
// It takes the well-formed case only.  Anything else -- invalid JSON, a
// shape serde rejects, an encoder limit, and a few legal but rare forms
// (duplicate keys, a "-0" usize, lone surrogate escapes, non-ASCII gate
// names, numbers that under- or overflow) -- returns DQ_ERR_DECODE, and the
// caller decodes the text with the Python decoder, which gives the exact
// error or result.  So every circuit this decoder accepts decodes the same
// way in both.
#include <charconv>
#include <cstdint>
#include <cstring>
#include <string>
#include <string_view>
#include <unordered_map>
#include <vector>

#include "dq_common.cuh"

struct dq_circuit {
  std::vector<dq_inst> insts;
  std::vector<dq_cond> conds;
  std::string names;  // packed (u64 index, u64 length, bytes) records
  uint64_t num_qubits = 0, num_cbits = 0, cbit_space = 1;
};

namespace dq {
namespace {

// ---- field tables (the variant tags and field orders of src/types.rs) ----

enum FieldType : uint8_t { F_U, F_F, F_S, F_FL, F_UL, F_COND, F_INST };

struct Field {
  const char* name;
  FieldType type;
};

struct Variant {
  const char* tag;
  int kind;  // enum dq_kind, or -1 for gate / conditional
  int nfields;
  Field f[6];
};

constexpr Field kQ{"qubit", F_U};
constexpr Field kCtl{"control", F_U};
constexpr Field kTgt{"target", F_U};

const Variant kVariants[] = {
    {"id", DQ_ID, 1, {kQ}},
    {"x", DQ_X, 1, {kQ}},
    {"y", DQ_Y, 1, {kQ}},
    {"z", DQ_Z, 1, {kQ}},
    {"h", DQ_H, 1, {kQ}},
    {"s", DQ_S, 1, {kQ}},
    {"sdg", DQ_SDG, 1, {kQ}},
    {"t", DQ_T, 1, {kQ}},
    {"tdg", DQ_TDG, 1, {kQ}},
    {"sx", DQ_SX, 1, {kQ}},
    {"sxdg", DQ_SXDG, 1, {kQ}},
    {"u0", DQ_U0, 1, {kQ}},
    {"reset", DQ_RESET, 1, {kQ}},
    {"u3", DQ_U3, 4, {kQ, {"theta", F_F}, {"phi", F_F}, {"lam", F_F}}},
    {"u", DQ_U, 4, {kQ, {"theta", F_F}, {"phi", F_F}, {"lam", F_F}}},
    {"u2", DQ_U2, 3, {kQ, {"phi", F_F}, {"lam", F_F}}},
    {"u1", DQ_U1, 2, {kQ, {"lam", F_F}}},
    {"p", DQ_P, 2, {kQ, {"lam", F_F}}},
    {"rx", DQ_RX, 2, {kQ, {"theta", F_F}}},
    {"ry", DQ_RY, 2, {kQ, {"theta", F_F}}},
    {"rz", DQ_RZ, 2, {kQ, {"phi", F_F}}},
    {"cx", DQ_CX, 2, {kCtl, kTgt}},
    {"cz", DQ_CZ, 2, {kCtl, kTgt}},
    {"cy", DQ_CY, 2, {kCtl, kTgt}},
    {"ch", DQ_CH, 2, {kCtl, kTgt}},
    {"csx", DQ_CSX, 2, {kCtl, kTgt}},
    {"swap", DQ_SWAP, 2, {{"a", F_U}, {"b", F_U}}},
    {"crx", DQ_CRX, 3, {kCtl, kTgt, {"theta", F_F}}},
    {"cry", DQ_CRY, 3, {kCtl, kTgt, {"theta", F_F}}},
    {"crz", DQ_CRZ, 3, {kCtl, kTgt, {"lam", F_F}}},
    {"cu1", DQ_CU1, 3, {kCtl, kTgt, {"lam", F_F}}},
    {"cp", DQ_CP, 3, {kCtl, kTgt, {"lam", F_F}}},
    {"cu3", DQ_CU3, 5, {kCtl, kTgt, {"theta", F_F}, {"phi", F_F}, {"lam", F_F}}},
    {"cu", DQ_CU, 6, {kCtl, kTgt, {"theta", F_F}, {"phi", F_F}, {"lam", F_F}, {"gamma", F_F}}},
    {"rxx", DQ_RXX, 3, {{"a", F_U}, {"b", F_U}, {"theta", F_F}}},
    {"rzz", DQ_RZZ, 3, {{"a", F_U}, {"b", F_U}, {"theta", F_F}}},
    {"ccx", DQ_CCX, 3, {{"control1", F_U}, {"control2", F_U}, kTgt}},
    {"rccx", DQ_RCCX, 3, {{"control1", F_U}, {"control2", F_U}, kTgt}},
    {"cswap", DQ_CSWAP, 3, {kCtl, {"target1", F_U}, {"target2", F_U}}},
    {"rc3x", DQ_RC3X, 4, {{"control1", F_U}, {"control2", F_U}, {"control3", F_U}, kTgt}},
    {"c3x", DQ_C3X, 4, {{"control1", F_U}, {"control2", F_U}, {"control3", F_U}, kTgt}},
    {"c3sqrtx", DQ_C3SQRTX, 4, {{"control1", F_U}, {"control2", F_U}, {"control3", F_U}, kTgt}},
    {"c4x", DQ_C4X, 5,
     {{"control1", F_U}, {"control2", F_U}, {"control3", F_U}, {"control4", F_U}, kTgt}},
    {"measure", DQ_MEASURE, 2, {kQ, {"cbit", F_U}}},
    {"barrier", DQ_BARRIER, 0, {}},
    {"classical", DQ_CLASSICAL, 1, {{"name", F_S}}},
    {"gate", -1, 3, {{"name", F_S}, {"params", F_FL}, {"qubits", F_UL}}},
    {"conditional", -1, 2, {{"condition", F_COND}, {"op", F_INST}}},
};

// generic `gate` names the dispatcher knows, lower-cased
// (statevector/simulator.rs:571-600 and 802-831)
struct Generic {
  const char* name;
  int kind;
};
const Generic kGeneric[] = {
    {"remote_link_phi_plus", DQ_G_PHI_PLUS}, {"remote_epr", DQ_G_PHI_PLUS},
    {"remote_link_psi_minus", DQ_G_PSI_MINUS}, {"remote_link_psi_plus", DQ_G_PSI_PLUS},
    {"nonlocal_cz", DQ_G_CZ}, {"remote_cz", DQ_G_CZ}, {"remote_cx", DQ_G_CX},
    {"remote_barrier", DQ_G_NOOP}, {"remote_cu1", DQ_G_NOOP},
};

// tag -> variant (built once; lookups are per instruction)
const Variant* variant(const std::string& tag) {
  static const std::unordered_map<std::string_view, const Variant*> table = [] {
    std::unordered_map<std::string_view, const Variant*> t;
    for (const auto& v : kVariants) t.emplace(v.tag, &v);
    return t;
  }();
  const auto it = table.find(std::string_view(tag));
  return it == table.end() ? nullptr : it->second;
}

constexpr uint64_t kMaxCbitSpace = 1ULL << 26;
constexpr uint64_t kMaxQubitIndex = 1ULL << 31;  // qubit fields at or above: encoder error

// ---- a strict reader over the JSON text ----------------------------------

struct Span {
  const char* b = nullptr;
  const char* e = nullptr;
};

struct Reader {
  const char* p;
  const char* end;

  void ws() {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
  }
  bool eat(char c) {
    ws();
    if (p < end && *p == c) {
      ++p;
      return true;
    }
    return false;
  }
  bool peek(char c) {
    ws();
    return p < end && *p == c;
  }

  // A JSON string into `out` (UTF-8).  Declines control characters and lone
  // surrogates.
  bool string(std::string& out) {
    ws();
    if (p >= end || *p != '"') return false;
    ++p;
    out.clear();
    // plain run up to the closing quote or the first escape, copied at once
    const char* run = p;
    while (p < end && *p != '"' && *p != '\\' && (unsigned char)*p >= 0x20) ++p;
    out.assign(run, p);
    while (p < end) {
      const unsigned char c = (unsigned char)*p++;
      if (c == '"') return true;
      if (c < 0x20) return false;
      if (c != '\\') {
        out.push_back((char)c);
        continue;
      }
      if (p >= end) return false;
      const char e = *p++;
      switch (e) {
        case '"': out.push_back('"'); break;
        case '\\': out.push_back('\\'); break;
        case '/': out.push_back('/'); break;
        case 'b': out.push_back('\b'); break;
        case 'f': out.push_back('\f'); break;
        case 'n': out.push_back('\n'); break;
        case 'r': out.push_back('\r'); break;
        case 't': out.push_back('\t'); break;
        case 'u': {
          uint32_t cp = 0;
          if (!hex4(cp)) return false;
          if (cp >= 0xD800 && cp <= 0xDBFF) {
            uint32_t lo = 0;
            if (end - p < 6 || p[0] != '\\' || p[1] != 'u') return false;
            p += 2;
            if (!hex4(lo) || lo < 0xDC00 || lo > 0xDFFF) return false;
            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
          } else if (cp >= 0xDC00 && cp <= 0xDFFF) {
            return false;
          }
          utf8(cp, out);
          break;
        }
        default: return false;
      }
    }
    return false;
  }
  bool hex4(uint32_t& v) {
    if (end - p < 4) return false;
    v = 0;
    for (int i = 0; i < 4; ++i) {
      const char c = *p++;
      v <<= 4;
      if (c >= '0' && c <= '9') v |= (uint32_t)(c - '0');
      else if (c >= 'a' && c <= 'f') v |= (uint32_t)(c - 'a' + 10);
      else if (c >= 'A' && c <= 'F') v |= (uint32_t)(c - 'A' + 10);
      else return false;
    }
    return true;
  }
  static void utf8(uint32_t cp, std::string& out) {
    if (cp < 0x80) {
      out.push_back((char)cp);
    } else if (cp < 0x800) {
      out.push_back((char)(0xC0 | (cp >> 6)));
      out.push_back((char)(0x80 | (cp & 0x3F)));
    } else if (cp < 0x10000) {
      out.push_back((char)(0xE0 | (cp >> 12)));
      out.push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
      out.push_back((char)(0x80 | (cp & 0x3F)));
    } else {
      out.push_back((char)(0xF0 | (cp >> 18)));
      out.push_back((char)(0x80 | ((cp >> 12) & 0x3F)));
      out.push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
      out.push_back((char)(0x80 | (cp & 0x3F)));
    }
  }

  // A JSON number token (RFC 8259 grammar); `integer` = no fraction or
  // exponent (Python's json yields an int for exactly these).
  bool number(Span& tok, bool& integer) {
    ws();
    const char* s = p;
    if (p < end && *p == '-') ++p;
    if (p >= end) return false;
    if (*p == '0') {
      ++p;
    } else if (*p >= '1' && *p <= '9') {
      while (p < end && *p >= '0' && *p <= '9') ++p;
    } else {
      return false;
    }
    integer = true;
    if (p < end && *p == '.') {
      ++p;
      if (p >= end || *p < '0' || *p > '9') return false;
      while (p < end && *p >= '0' && *p <= '9') ++p;
      integer = false;
    }
    if (p < end && (*p == 'e' || *p == 'E')) {
      ++p;
      if (p < end && (*p == '+' || *p == '-')) ++p;
      if (p >= end || *p < '0' || *p > '9') return false;
      while (p < end && *p >= '0' && *p <= '9') ++p;
      integer = false;
    }
    // very long tokens (Python's int conversion caps the digit count) are
    // left to the full decoder
    if (p - s > 1000) return false;
    tok.b = s;
    tok.e = p;
    return true;
  }

  bool literal(const char* w) {
    const size_t n = strlen(w);
    if ((size_t)(end - p) < n || memcmp(p, w, n) != 0) return false;
    p += n;
    return true;
  }

  // Skip one value of any type (validating it), depth-limited.
  bool skip(int depth = 0) {
    if (depth > 64) return false;
    ws();
    if (p >= end) return false;
    const char c = *p;
    if (c == '"') {
      std::string tmp;
      return string(tmp);
    }
    if (c == '{') {
      ++p;
      if (eat('}')) return true;
      std::string key;
      do {
        if (!string(key) || !eat(':') || !skip(depth + 1)) return false;
      } while (eat(','));
      return eat('}');
    }
    if (c == '[') {
      ++p;
      if (eat(']')) return true;
      do {
        if (!skip(depth + 1)) return false;
      } while (eat(','));
      return eat(']');
    }
    if (c == 't') return literal("true");
    if (c == 'f') return literal("false");
    if (c == 'n') return literal("null");
    Span t;
    bool integer;
    return number(t, integer);
  }

  // Visit the members of an object: fn(key) consumes the value.  Declines a
  // key seen twice (Python keeps the last; serde reports the duplicate).
  template <class Fn>
  bool object(Fn&& fn) {
    if (!eat('{')) return false;
    if (eat('}')) return true;
    constexpr int kMaxKeys = 24;  // more members: left to the full decoder
    std::string seen[kMaxKeys];
    int nseen = 0;
    std::string key;
    do {
      if (!string(key) || !eat(':') || nseen == kMaxKeys) return false;
      for (int i = 0; i < nseen; ++i)
        if (seen[i] == key) return false;
      seen[nseen++] = key;
      if (!fn(key)) return false;
    } while (eat(','));
    return eat('}');
  }
};

// usize: a non-negative JSON integer that fits 64 bits ("-0" is left to the
// full decoder).
bool to_usize(Span t, bool integer, uint64_t& v) {
  if (!integer || *t.b == '-') return false;
  auto r = std::from_chars(t.b, t.e, v);
  return r.ec == std::errc() && r.ptr == t.e;
}

// f64: a JSON integer or float, finite after correctly rounded conversion
// (Python's float()); an integer keeps the sign of zero out, as float(int).
bool to_f64(Span t, bool integer, double& v) {
  auto r = std::from_chars(t.b, t.e, v);
  if (r.ec != std::errc() || r.ptr != t.e) return false;
  if (!(v - v == 0.0)) return false;  // inf / nan
  if (integer && v == 0.0) v = 0.0;
  return true;
}

struct Decoder {
  Reader rd;
  dq_circuit* c;
  uint64_t max_cbit_plus1 = 0;  // highest classical bit referenced + 1

  bool usize(uint64_t& v) {
    Span t;
    bool integer;
    return rd.number(t, integer) && to_usize(t, integer, v);
  }
  bool f64(double& v) {
    Span t;
    bool integer;
    return rd.number(t, integer) && to_f64(t, integer, v);
  }

  bool registers(uint64_t& width) {
    width = 0;
    return rd.object([&](const std::string&) {
      bool has_name = false, has_size = false, has_base = false;
      uint64_t size = 0, base = 0;
      std::string name;
      if (!rd.object([&](const std::string& k) {
            if (k == "name") return (has_name = true) && rd.string(name);
            if (k == "size") return (has_size = true) && usize(size);
            if (k == "base") return (has_base = true) && usize(base);
            return rd.skip();
          }))
        return false;
      if (!has_name || !has_size || !has_base) return false;
      if (base + size < base) return false;  // wider than 64 bits
      if (base + size > width) width = base + size;
      return true;
    });
  }

  // One instruction object, appended to c->insts with its condition chain.
  // The object's members come in any order; the tag decides which are read,
  // so the members are first located and then decoded.
  bool instruction(uint64_t idx, std::vector<dq_cond>& chain, int depth) {
    if (depth > 32) return false;
    struct Member {
      std::string key;
      const char* at;
    };
    constexpr int kMaxMembers = 24;  // the object reader's own limit
    Member members[kMaxMembers];
    int nm = 0;
    if (!rd.object([&](const std::string& k) {
          rd.ws();
          members[nm].key = k;
          members[nm++].at = rd.p;
          return rd.skip();
        }))
      return false;
    const char* after = rd.p;
    const char* tag_at = nullptr;
    for (int i = 0; i < nm; ++i)
      if (members[i].key == "kind") tag_at = members[i].at;
    if (!tag_at) return false;
    std::string tag;
    rd.p = tag_at;
    if (!rd.string(tag)) return false;
    const Variant* v = variant(tag);
    if (!v) return false;
    auto find = [&](const char* name) -> const char* {
      for (int i = 0; i < nm; ++i)
        if (members[i].key == name) return members[i].at;
      return nullptr;
    };
    for (int i = 0; i < v->nfields; ++i)
      if (!find(v->f[i].name)) return false;

    if (tag == "conditional") {
      dq_cond cd{0, 0, 0};
      bool hb = false, hs = false, hv = false;
      rd.p = find("condition");
      if (!rd.object([&](const std::string& k) {
            if (k == "creg_base") return (hb = true) && usize(cd.creg_base);
            if (k == "creg_size") return (hs = true) && usize(cd.creg_size);
            if (k == "creg_value") return (hv = true) && usize(cd.creg_value);
            return rd.skip();
          }))
        return false;
      if (!hb || !hs || !hv) return false;
      chain.push_back(cd);
      rd.p = find("op");
      const bool ok = instruction(idx, chain, depth + 1);
      chain.pop_back();
      rd.p = after;
      return ok;
    }

    dq_inst in;
    memset(&in, 0, sizeof(in));
    for (int i = 0; i < DQ_MAX_INST_QUBITS; ++i) in.q[i] = -1;
    if (tag == "gate") {
      std::string name;
      rd.p = find("name");
      if (!rd.string(name)) return false;
      for (auto& ch : name) {
        if ((unsigned char)ch >= 0x80) return false;  // Unicode lower-casing: full decoder
        if (ch >= 'A' && ch <= 'Z') ch = (char)(ch - 'A' + 'a');
      }
      rd.p = find("params");
      if (!rd.eat('[')) return false;
      if (!rd.eat(']')) {
        do {
          double x;
          if (!f64(x)) return false;
        } while (rd.eat(','));
        if (!rd.eat(']')) return false;
      }
      std::vector<uint64_t> qs;
      rd.p = find("qubits");
      if (!rd.eat('[')) return false;
      if (!rd.eat(']')) {
        do {
          uint64_t q;
          if (!usize(q)) return false;
          qs.push_back(q);
        } while (rd.eat(','));
        if (!rd.eat(']')) return false;
      }
      int kind = DQ_G_UNSUPPORTED;
      for (const auto& g : kGeneric)
        if (name == g.name) kind = g.kind;
      if (kind == DQ_G_UNSUPPORTED && name.compare(0, 8, "circuit-") == 0) kind = DQ_G_OPAQUE;
      in.kind = kind;
      const bool two = kind == DQ_G_PHI_PLUS || kind == DQ_G_PSI_MINUS || kind == DQ_G_PSI_PLUS ||
                       kind == DQ_G_CZ || kind == DQ_G_CX;
      if (two && qs.size() != 2) return false;  // encoder error: full decoder reports it
      const size_t nq = qs.size() < DQ_MAX_INST_QUBITS ? qs.size() : DQ_MAX_INST_QUBITS;
      in.nq = (int32_t)nq;
      for (size_t i = 0; i < nq; ++i) in.q[i] = qs[i] < kMaxQubitIndex ? (int32_t)qs[i] : -1;
      const uint64_t len = name.size();
      c->names.append(reinterpret_cast<const char*>(&idx), 8);
      c->names.append(reinterpret_cast<const char*>(&len), 8);
      c->names.append(name);
    } else {
      in.kind = v->kind;
      int nq = 0, np = 0;
      for (int i = 0; i < v->nfields; ++i) {
        const Field& f = v->f[i];
        rd.p = find(f.name);
        if (f.type == F_U) {
          uint64_t x;
          if (!usize(x)) return false;
          if (v->kind == DQ_MEASURE && strcmp(f.name, "cbit") == 0) {
            if (x >= kMaxCbitSpace) return false;  // classical space limit
            in.cbit = (int64_t)x;
            if (x + 1 > max_cbit_plus1) max_cbit_plus1 = x + 1;
          } else {
            if (x >= kMaxQubitIndex) return false;
            in.q[nq++] = (int32_t)x;
          }
        } else if (f.type == F_F) {
          if (!f64(in.p[np++])) return false;
        } else {  // F_S: classical name
          std::string s;
          if (!rd.string(s)) return false;
        }
      }
      in.nq = (v->kind == DQ_BARRIER || v->kind == DQ_CLASSICAL) ? 0 : nq;
    }
    if (!chain.empty()) {
      in.cond_first = (uint32_t)c->conds.size();
      in.cond_count = (uint32_t)chain.size();
      for (const auto& cd : chain) {
        if (cd.creg_size > 64) return false;
        if (cd.creg_size > 0) {
          const uint64_t top = cd.creg_base + cd.creg_size;  // highest bit + 1
          if (top < cd.creg_base || top > kMaxCbitSpace) return false;
          if (top > max_cbit_plus1) max_cbit_plus1 = top;
        }
        c->conds.push_back(cd);
      }
    }
    c->insts.push_back(in);
    rd.p = after;
    return true;
  }

  bool circuit() {
    bool has_q = false, has_c = false, has_i = false;
    uint64_t nq = 0, nc = 0;
    if (!rd.object([&](const std::string& k) {
          if (k == "qregs") return (has_q = true) && registers(nq);
          if (k == "cregs") return (has_c = true) && registers(nc);
          if (k == "instructions") {
            has_i = true;
            if (!rd.eat('[')) return false;
            if (rd.eat(']')) return true;
            std::vector<dq_cond> chain;
            do {
              rd.ws();
              if (!instruction(c->insts.size(), chain, 0)) return false;
            } while (rd.eat(','));
            return rd.eat(']');
          }
          return rd.skip();
        }))
      return false;
    rd.ws();
    if (rd.p != rd.end || !has_q || !has_i) return false;
    (void)has_c;
    c->num_qubits = nq;
    c->num_cbits = nc;
    uint64_t space = nc > max_cbit_plus1 ? nc : max_cbit_plus1;
    if (space < 1) space = 1;
    if (space > kMaxCbitSpace) return false;
    c->cbit_space = space;
    return true;
  }
};

}  // namespace
}  // namespace dq

extern "C" {

int dq_circuit_decode(const char* json, uint64_t len, dq_circuit** out, dq_circuit_info* info) {
  if (!out || !info || (len && !json)) return dq::fail(DQ_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  dq_circuit* c = new (std::nothrow) dq_circuit();
  if (!c) return dq::fail(DQ_ERR_OOM, "dq_circuit_decode: out of host memory");
  dq::Decoder d{dq::Reader{json, json + len}, c};
  bool ok = false;
  try {
    ok = d.circuit();
  } catch (const std::bad_alloc&) {
    delete c;
    return dq::fail(DQ_ERR_OOM, "dq_circuit_decode: out of host memory");
  }
  if (!ok) {
    const uint64_t at = (uint64_t)(d.rd.p - json);
    delete c;
    return dq::fail(DQ_ERR_DECODE, "circuit JSON not decoded natively (near byte " +
                                       std::to_string(at) + ")");
  }
  info->ninst = c->insts.size();
  info->ncond = c->conds.size();
  info->num_qubits = c->num_qubits;
  info->num_cbits = c->num_cbits;
  info->cbit_space = c->cbit_space;
  info->names_bytes = c->names.size();
  *out = c;
  return DQ_OK;
}

int dq_circuit_export(const dq_circuit* c, dq_inst* insts, dq_cond* conds, uint8_t* names) {
  if (!c) return dq::fail(DQ_ERR_INVALID_ARG, "null circuit");
  if ((!c->insts.empty() && !insts) || (!c->conds.empty() && !conds) ||
      (!c->names.empty() && !names))
    return dq::fail(DQ_ERR_INVALID_ARG, "null output buffer");
  if (!c->insts.empty()) memcpy(insts, c->insts.data(), sizeof(dq_inst) * c->insts.size());
  if (!c->conds.empty()) memcpy(conds, c->conds.data(), sizeof(dq_cond) * c->conds.size());
  if (!c->names.empty()) memcpy(names, c->names.data(), c->names.size());
  return DQ_OK;
}

void dq_circuit_free(dq_circuit* c) { delete c; }

}  // extern "C"
