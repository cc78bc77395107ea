// persist.cpp — gprx's on-disk model format (format_version 1) for exact
// models: a directory with config.json (what the model is) and
// model.safetensors (x, y and, saved with the factor, l and alpha).
//
// The format is gprx's (docs/persist-format.md; src/persist/mod.rs,
// src/persist/tensors.rs, src/persist/kernel.rs): JSON with serde's external
// tagging, bounded parameters {"value", "lo", "hi"}, matrices column-major
// under a row-major-looking [rows, cols] shape, tensor bytes 8-byte aligned.
// This backend reads and writes the part of it that its kernels cover: the
// rbf / rbf_ard / constant / periodic leaves under sum / product, identity
// input and target maps, double precision, llt and ldlt factors.  Anything
// else is refused with GPRX_PERSIST_FAILED and a message naming it.
//
// Host code only: a small JSON reader/writer and the safetensors layout.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "persist.h"

namespace gprx {

// the per-thread error record of the library (capi.cu)
gprx_status set_error(gprx_status st, const std::string& msg);

// ---------------------------------------------------------------------------
// JSON
// ---------------------------------------------------------------------------
struct Json {
  enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<Json> arr;
  std::vector<std::pair<std::string, Json>> obj;  // insertion order (the writer keeps it)

  const Json* get(const std::string& k) const {
    if (kind != OBJ) return nullptr;
    for (auto& kv : obj)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
  Json& set(const std::string& k, Json v) {
    obj.emplace_back(k, std::move(v));
    return obj.back().second;
  }
  static Json number(double v) {
    Json j;
    j.kind = NUM;
    j.num = v;
    return j;
  }
  static Json string(const std::string& s) {
    Json j;
    j.kind = STR;
    j.str = s;
    return j;
  }
  static Json boolean(bool v) {
    Json j;
    j.kind = BOOL;
    j.b = v;
    return j;
  }
  static Json object() {
    Json j;
    j.kind = OBJ;
    return j;
  }
  static Json array() {
    Json j;
    j.kind = ARR;
    return j;
  }
};

struct JsonParser {
  const char* p;
  const char* end;
  int depth = 0;
  std::string err;

  void ws() {
    while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
  }
  bool fail(const char* why) {
    if (err.empty()) err = why;
    return false;
  }
  bool lit(const char* s) {
    size_t n = std::strlen(s);
    if ((size_t)(end - p) < n || std::strncmp(p, s, n) != 0) return false;
    p += n;
    return true;
  }
  bool str(std::string& out) {
    if (p >= end || *p != '"') return fail("expected a string");
    ++p;
    out.clear();
    while (p < end && *p != '"') {
      if (*p == '\\') {
        ++p;
        if (p >= end) return fail("bad escape");
        char c = *p++;
        switch (c) {
          case '"': out += '"'; break;
          case '\\': out += '\\'; break;
          case '/': out += '/'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'n': out += '\n'; break;
          case 'r': out += '\r'; break;
          case 't': out += '\t'; break;
          case 'u': {
            if (end - p < 4) return fail("bad \\u escape");
            unsigned v = 0;
            for (int i = 0; i < 4; ++i) {
              char h = *p++;
              v <<= 4;
              if (h >= '0' && h <= '9') v |= h - '0';
              else if (h >= 'a' && h <= 'f') v |= h - 'a' + 10;
              else if (h >= 'A' && h <= 'F') v |= h - 'A' + 10;
              else return fail("bad \\u escape");
            }
            // UTF-8 of a BMP code point (surrogate pairs are not needed by the format's keys)
            if (v < 0x80) out += (char)v;
            else if (v < 0x800) { out += (char)(0xC0 | (v >> 6)); out += (char)(0x80 | (v & 0x3F)); }
            else { out += (char)(0xE0 | (v >> 12)); out += (char)(0x80 | ((v >> 6) & 0x3F)); out += (char)(0x80 | (v & 0x3F)); }
            break;
          }
          default: return fail("bad escape");
        }
      } else {
        out += *p++;
      }
    }
    if (p >= end) return fail("unterminated string");
    ++p;
    return true;
  }
  bool value(Json& v) {
    ws();
    if (p >= end) return fail("unexpected end of JSON");
    if (++depth > 128) return fail("JSON nested deeper than 128");
    bool ok = true;
    if (*p == '{') {
      ++p;
      v = Json::object();
      ws();
      if (p < end && *p == '}') {
        ++p;
      } else {
        for (;;) {
          ws();
          std::string k;
          if (!str(k)) { ok = false; break; }
          ws();
          if (p >= end || *p != ':') { ok = fail("expected ':'"); break; }
          ++p;
          Json c;
          if (!value(c)) { ok = false; break; }
          v.obj.emplace_back(std::move(k), std::move(c));
          ws();
          if (p < end && *p == ',') { ++p; continue; }
          if (p < end && *p == '}') { ++p; break; }
          ok = fail("expected ',' or '}'");
          break;
        }
      }
    } else if (*p == '[') {
      ++p;
      v = Json::array();
      ws();
      if (p < end && *p == ']') {
        ++p;
      } else {
        for (;;) {
          Json c;
          if (!value(c)) { ok = false; break; }
          v.arr.push_back(std::move(c));
          ws();
          if (p < end && *p == ',') { ++p; continue; }
          if (p < end && *p == ']') { ++p; break; }
          ok = fail("expected ',' or ']'");
          break;
        }
      }
    } else if (*p == '"') {
      v.kind = Json::STR;
      ok = str(v.str);
    } else if (lit("true")) {
      v = Json::boolean(true);
    } else if (lit("false")) {
      v = Json::boolean(false);
    } else if (lit("null")) {
      v = Json();
    } else {
      // strtod rounds correctly, so a number written in its shortest
      // round-trip form comes back to the bit
      char* e = nullptr;
      std::string tok;
      const char* q = p;
      while (q < end && (std::strchr("+-0123456789.eE", *q) != nullptr)) ++q;
      tok.assign(p, q);
      double d = std::strtod(tok.c_str(), &e);
      if (tok.empty() || e != tok.c_str() + tok.size()) {
        ok = fail("bad JSON value");
      } else {
        v = Json::number(d);
        p = q;
      }
    }
    --depth;
    return ok;
  }
};

static bool parse_json(const std::string& text, Json& out, std::string& err) {
  JsonParser ps{text.data(), text.data() + text.size()};
  if (!ps.value(out)) {
    err = ps.err;
    return false;
  }
  ps.ws();
  if (ps.p != ps.end) {
    err = "trailing characters after the JSON value";
    return false;
  }
  return true;
}

static std::string fmt_num(double v) {
  // the shortest of %.15g / %.16g / %.17g that reads back to the same bits
  char buf[40];
  for (int prec = 15; prec <= 17; ++prec) {
    std::snprintf(buf, sizeof buf, "%.*g", prec, v);
    if (std::strtod(buf, nullptr) == v) break;
  }
  std::string s(buf);
  if (s.find_first_of(".eEn") == std::string::npos) s += ".0";  // keep it a float
  return s;
}

static void write_json(const Json& v, std::string& out, int indent) {
  const std::string pad((size_t)indent * 2, ' '), pad2((size_t)(indent + 1) * 2, ' ');
  switch (v.kind) {
    case Json::NUL: out += "null"; break;
    case Json::BOOL: out += v.b ? "true" : "false"; break;
    case Json::NUM: out += fmt_num(v.num); break;
    case Json::STR: {
      out += '"';
      for (char c : v.str) {
        if (c == '"' || c == '\\') { out += '\\'; out += c; }
        else if (c == '\n') out += "\\n";
        else out += c;
      }
      out += '"';
      break;
    }
    case Json::ARR: {
      if (v.arr.empty()) { out += "[]"; break; }
      out += "[\n";
      for (size_t i = 0; i < v.arr.size(); ++i) {
        out += pad2;
        write_json(v.arr[i], out, indent + 1);
        out += i + 1 < v.arr.size() ? ",\n" : "\n";
      }
      out += pad + "]";
      break;
    }
    case Json::OBJ: {
      if (v.obj.empty()) { out += "{}"; break; }
      out += "{\n";
      for (size_t i = 0; i < v.obj.size(); ++i) {
        out += pad2 + "\"" + v.obj[i].first + "\": ";
        write_json(v.obj[i].second, out, indent + 1);
        out += i + 1 < v.obj.size() ? ",\n" : "\n";
      }
      out += pad + "}";
      break;
    }
  }
}

static Json json_int(long long v) {
  Json j = Json::number((double)v);
  return j;
}

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static gprx_status pfail(const std::string& kind, const std::string& why) {
  return set_error(GPRX_PERSIST_FAILED, "persist (" + kind + "): " + why);
}

// ---------------------------------------------------------------------------
// files
// ---------------------------------------------------------------------------
static bool read_file(const std::string& path, std::string& out) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  out.resize(sz > 0 ? (size_t)sz : 0);
  size_t got = sz > 0 ? std::fread(&out[0], 1, (size_t)sz, f) : 0;
  std::fclose(f);
  return got == out.size();
}

// written to a temporary name in the directory and renamed over the target
static bool write_file_atomic(const std::string& dir, const std::string& name, const std::string& data) {
  const std::string tmp = dir + "/." + name + ".tmp";
  FILE* f = std::fopen(tmp.c_str(), "wb");
  if (!f) return false;
  bool ok = std::fwrite(data.data(), 1, data.size(), f) == data.size();
  ok = (std::fflush(f) == 0) && ok;
  ok = (fsync(fileno(f)) == 0) && ok;
  std::fclose(f);
  if (!ok || std::rename(tmp.c_str(), (dir + "/" + name).c_str()) != 0) {
    std::remove(tmp.c_str());
    return false;
  }
  return true;
}

static bool make_dirs(const std::string& dir) {
  std::string cur;
  for (size_t i = 0; i <= dir.size(); ++i) {
    if (i == dir.size() || dir[i] == '/') {
      if (!cur.empty() && cur != "/") {
        if (mkdir(cur.c_str(), 0777) != 0 && errno != EEXIST) return false;
      }
    }
    if (i < dir.size()) cur += dir[i];
  }
  struct stat st;
  return stat(dir.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

// ---------------------------------------------------------------------------
// kernel tree <-> JSON (src/persist/kernel.rs)
// ---------------------------------------------------------------------------
static const double LO = 1e-5, HI = 1e5;  // Interval::DEFAULT_POSITIVE (src/param.rs:91)

static Json bounded(double v) {
  Json b = Json::object();
  b.set("value", Json::number(v));
  b.set("lo", Json::number(LO));
  b.set("hi", Json::number(HI));
  return b;
}

static bool read_bounded(const Json* b, double& v, std::string& why) {
  const Json* val = b ? b->get("value") : nullptr;
  const Json* lo = b ? b->get("lo") : nullptr;
  const Json* hi = b ? b->get("hi") : nullptr;
  if (!val || val->kind != Json::NUM || !lo || lo->kind != Json::NUM || !hi || hi->kind != Json::NUM) {
    why = "a bounded parameter needs numeric value, lo and hi";
    return false;
  }
  if (!std::isfinite(lo->num) || !std::isfinite(hi->num) || !(lo->num < hi->num) || !std::isfinite(val->num) ||
      !(val->num > lo->num && val->num < hi->num)) {
    why = "a bounded parameter is outside its interval";
    return false;
  }
  v = val->num;
  return true;
}

// prefix nodes [i, …) → JSON; θ (log) consumed in depth-first order
static Json encode_kernel(const std::vector<gprx_kernel_node>& nodes, size_t& i, const double* theta, size_t& t) {
  const gprx_kernel_node nd = nodes[i++];
  if (nd.kind == GPRX_NODE_SUM || nd.kind == GPRX_NODE_PRODUCT) {
    const char* tag = nd.kind == GPRX_NODE_SUM ? "sum" : "product";
    Json acc = encode_kernel(nodes, i, theta, t);
    for (int c = 1; c < nd.arg; ++c) {  // n-ary → left-nested binary (θ order kept)
      Json right = encode_kernel(nodes, i, theta, t);
      Json body = Json::object();
      body.set("left", std::move(acc));
      body.set("right", std::move(right));
      acc = Json::object();
      acc.set(tag, std::move(body));
    }
    return acc;
  }
  Json leaf = Json::object(), body = Json::object();
  switch (nd.kind) {
    case GPRX_LEAF_RBF:
      body.set("lengthscale", bounded(std::exp(theta[t++])));
      leaf.set("rbf", std::move(body));
      break;
    case GPRX_LEAF_RBF_ARD: {
      Json ls = Json::array();
      for (int f = 0; f < nd.arg; ++f) ls.arr.push_back(bounded(std::exp(theta[t++])));
      body.set("lengthscales", std::move(ls));
      leaf.set("rbf_ard", std::move(body));
      break;
    }
    case GPRX_LEAF_CONSTANT:
      body.set("constant", bounded(std::exp(theta[t++])));
      leaf.set("constant", std::move(body));
      break;
    default:  // GPRX_LEAF_PERIODIC
      body.set("lengthscale", bounded(std::exp(theta[t++])));
      body.set("period", bounded(std::exp(theta[t++])));
      leaf.set("periodic", std::move(body));
      break;
  }
  return leaf;
}

// JSON → prefix nodes (chains of the same sum / product flattened) and θ
static bool decode_kernel(const Json& k, std::vector<gprx_kernel_node>& nodes, std::vector<double>& theta,
                          std::string& why) {
  if (k.kind != Json::OBJ || k.obj.size() != 1) {
    why = "a kernel is an object with one tag";
    return false;
  }
  const std::string& tag = k.obj[0].first;
  const Json& body = k.obj[0].second;
  if (tag == "sum" || tag == "product") {
    const int kind = tag == "sum" ? GPRX_NODE_SUM : GPRX_NODE_PRODUCT;
    std::vector<const Json*> kids;
    // in-order leaves of the same-tag chain, left to right
    std::function<bool(const Json&)> collect = [&](const Json& e) -> bool {
      if (e.kind == Json::OBJ && e.obj.size() == 1 && e.obj[0].first == tag) {
        const Json* l = e.obj[0].second.get("left");
        const Json* r = e.obj[0].second.get("right");
        if (!l || !r) {
          why = tag + " needs left and right";
          return false;
        }
        return collect(*l) && collect(*r);
      }
      kids.push_back(&e);
      return true;
    };
    if (!collect(k)) return false;
    nodes.push_back({kind, (int32_t)kids.size()});
    for (const Json* c : kids)
      if (!decode_kernel(*c, nodes, theta, why)) return false;
    return true;
  }
  double v = 0.0;
  if (tag == "rbf") {
    if (!read_bounded(body.get("lengthscale"), v, why)) return false;
    nodes.push_back({GPRX_LEAF_RBF, 0});
    theta.push_back(std::log(v));
  } else if (tag == "rbf_ard") {
    const Json* ls = body.get("lengthscales");
    if (!ls || ls->kind != Json::ARR) {
      why = "rbf_ard needs lengthscales";
      return false;
    }
    if (ls->arr.empty()) {
      why = "empty lengthscales";
      return false;
    }
    nodes.push_back({GPRX_LEAF_RBF_ARD, (int32_t)ls->arr.size()});
    for (auto& e : ls->arr) {
      if (!read_bounded(&e, v, why)) return false;
      theta.push_back(std::log(v));
    }
  } else if (tag == "constant") {
    if (!read_bounded(body.get("constant"), v, why)) return false;
    nodes.push_back({GPRX_LEAF_CONSTANT, 0});
    theta.push_back(std::log(v));
  } else if (tag == "periodic") {
    double p = 0.0;
    if (!read_bounded(body.get("lengthscale"), v, why) || !read_bounded(body.get("period"), p, why)) return false;
    nodes.push_back({GPRX_LEAF_PERIODIC, 0});
    theta.push_back(std::log(v));
    theta.push_back(std::log(p));
  } else {
    why = "kernel '" + tag + "' is not supported by this backend";
    return false;
  }
  return true;
}

// ---------------------------------------------------------------------------
// safetensors (src/persist/tensors.rs): 8-byte little-endian header length,
// JSON header {name: {dtype, shape, data_offsets}}, then the bytes
// ---------------------------------------------------------------------------
struct TensorOut {
  std::string name;
  std::vector<long long> shape;
  const double* data;
  size_t count;
};

static std::string safetensors_bytes(const std::vector<TensorOut>& ts) {
  Json h = Json::object();
  size_t off = 0;
  for (auto& t : ts) {
    Json e = Json::object();
    e.set("dtype", Json::string("F64"));
    Json sh = Json::array();
    for (long long s : t.shape) sh.arr.push_back(json_int(s));
    e.set("shape", std::move(sh));
    Json offs = Json::array();
    offs.arr.push_back(json_int((long long)off));
    offs.arr.push_back(json_int((long long)(off + t.count * 8)));
    e.set("data_offsets", std::move(offs));
    h.set(t.name, std::move(e));
    off += t.count * 8;
  }
  // compact header (integers written without a fraction)
  std::string hj = "{";
  for (size_t i = 0; i < h.obj.size(); ++i) {
    const auto& e = h.obj[i].second;
    hj += "\"" + h.obj[i].first + "\":{\"dtype\":\"F64\",\"shape\":[";
    const auto& sh = e.get("shape")->arr;
    for (size_t k = 0; k < sh.size(); ++k) hj += (k ? "," : "") + std::to_string((long long)sh[k].num);
    const auto& of = e.get("data_offsets")->arr;
    hj += "],\"data_offsets\":[" + std::to_string((long long)of[0].num) + "," + std::to_string((long long)of[1].num) +
          "]}";
    hj += i + 1 < h.obj.size() ? "," : "";
  }
  hj += "}";
  while ((8 + hj.size()) % 8 != 0) hj += ' ';  // tensor bytes 8-byte aligned
  std::string out(8, '\0');
  uint64_t hl = hj.size();
  for (int b = 0; b < 8; ++b) out[b] = (char)((hl >> (8 * b)) & 0xFF);
  out += hj;
  for (auto& t : ts) out.append(reinterpret_cast<const char*>(t.data), t.count * 8);
  return out;
}

// A read-only mapping of model.safetensors; tensors point into it.
struct Mapped {
  void* base = nullptr;
  size_t size = 0;
  ~Mapped() {
    if (base) munmap(base, size);
  }
};

struct TensorIn {
  const double* data = nullptr;
  std::vector<long long> shape;
  size_t count = 0;
};

static gprx_status map_safetensors(const std::string& path, Mapped& m, std::map<std::string, TensorIn>& out) {
  int fd = open(path.c_str(), O_RDONLY);
  if (fd < 0) return pfail("Io", "cannot open " + path);
  struct stat st;
  if (fstat(fd, &st) != 0 || st.st_size < 8) {
    close(fd);
    return pfail("Tensor", "model.safetensors is too short");
  }
  m.size = (size_t)st.st_size;
  m.base = mmap(nullptr, m.size, PROT_READ, MAP_PRIVATE, fd, 0);
  close(fd);
  if (m.base == MAP_FAILED) {
    m.base = nullptr;
    return pfail("Io", "cannot map " + path);
  }
  const unsigned char* b = (const unsigned char*)m.base;
  uint64_t hl = 0;
  for (int i = 0; i < 8; ++i) hl |= (uint64_t)b[i] << (8 * i);
  if (hl > m.size - 8) return pfail("Tensor", "safetensors header length past the end of the file");
  Json h;
  std::string err;
  if (!parse_json(std::string((const char*)b + 8, hl), h, err) || h.kind != Json::OBJ)
    return pfail("Tensor", "safetensors header: " + err);
  const size_t body = 8 + hl;
  for (auto& kv : h.obj) {
    if (kv.first == "__metadata__") continue;
    const Json* dt = kv.second.get("dtype");
    const Json* sh = kv.second.get("shape");
    const Json* of = kv.second.get("data_offsets");
    if (!dt || dt->kind != Json::STR || !sh || sh->kind != Json::ARR || !of || of->kind != Json::ARR ||
        of->arr.size() != 2)
      return pfail("Tensor", "tensor '" + kv.first + "' has no dtype / shape / data_offsets");
    if (dt->str != "F64") return pfail("Tensor", "tensor '" + kv.first + "' is " + dt->str + ", this backend reads F64");
    TensorIn t;
    size_t cnt = 1;
    for (auto& s : sh->arr) {
      if (s.kind != Json::NUM || s.num < 0) return pfail("Tensor", "bad shape of '" + kv.first + "'");
      t.shape.push_back((long long)s.num);
      cnt *= (size_t)s.num;
    }
    const size_t lo = (size_t)of->arr[0].num, hi = (size_t)of->arr[1].num;
    if (hi < lo || hi - lo != cnt * 8 || body + hi > m.size)
      return pfail("Tensor", "data_offsets of '" + kv.first + "' do not match its shape");
    if ((body + lo) % 8 != 0) return pfail("Tensor", "tensor '" + kv.first + "' is not 8-byte aligned");
    t.data = (const double*)(b + body + lo);
    t.count = cnt;
    for (size_t i = 0; i < cnt; ++i)
      if (!std::isfinite(t.data[i])) return pfail("Tensor", "tensor '" + kv.first + "' holds a non-finite value");
    out[kv.first] = t;
  }
  return GPRX_OK;
}

// ---------------------------------------------------------------------------
// model <-> directory
// ---------------------------------------------------------------------------
gprx_status persist_write(const std::string& dir, const PersistModel& m) {
  if (m.n <= 0 || m.d <= 0) return set_error(GPRX_EMPTY_INPUT, "persist: empty model");
  if (!make_dirs(dir)) return pfail("Io", "cannot create " + dir);
  Json c = Json::object();
  c.set("format_version", json_int(1));
  c.set("n", json_int(m.n));
  c.set("d", json_int(m.d));
  c.set("has_factor", Json::boolean(m.has_factor));
  c.set("factor_kind", Json::string(m.ldlt ? "ldlt" : "llt"));
  size_t i = 0, t = 0;
  c.set("kernel", encode_kernel(m.nodes, i, m.theta.data(), t));
  Json lik = Json::object();
  lik.set("noise_variance", bounded(std::exp(m.log_noise)));
  c.set("likelihood", std::move(lik));
  Json jit = Json::object();
  if (m.jitter.jitter_kind == GPRX_JITTER_FIXED) {
    Json f = Json::object();
    f.set("jitter", Json::number(m.jitter.jitter_initial));
    jit.set("fixed", std::move(f));
  } else {
    Json a = Json::object();
    a.set("initial", Json::number(m.jitter.jitter_initial));
    a.set("multiplier", Json::number(m.jitter.jitter_multiplier));
    a.set("max_retries", json_int(m.jitter.jitter_max_retries));
    a.set("max_jitter", Json::number(m.jitter.jitter_max));
    jit.set("adaptive", std::move(a));
  }
  c.set("jitter", std::move(jit));
  if (m.has_factor && m.factor_jitter != 0.0) c.set("factor_jitter", Json::number(m.factor_jitter));
  c.set("distance_cache", Json::string("always"));
  c.set("x_unfitted", Json::string("identity"));
  c.set("y_unfitted", Json::string("identity"));
  c.set("x_transform", Json::string("identity"));
  c.set("y_transform", Json::string("identity"));
  if (m.ldlt) {
    Json ids = Json::array();
    for (uint64_t id : m.ids) ids.arr.push_back(json_int((long long)id));
    c.set("point_ids", std::move(ids));
    c.set("next_point_id", json_int((long long)m.next_id));
  }
  std::vector<TensorOut> ts;
  ts.push_back({"x", {m.n, m.d}, m.x.data(), m.x.size()});
  ts.push_back({"y", {m.n}, m.y.data(), m.y.size()});
  if (m.has_factor) {
    ts.push_back({"l", {m.n, m.n}, m.l.data(), m.l.size()});
    ts.push_back({"alpha", {m.n}, m.alpha.data(), m.alpha.size()});
  }
  std::string cfg;
  write_json(c, cfg, 0);
  cfg += "\n";
  // the tensors first and the config last: a reader sees the old model or the new one
  if (!write_file_atomic(dir, "model.safetensors", safetensors_bytes(ts)))
    return pfail("Io", "cannot write " + dir + "/model.safetensors");
  if (!write_file_atomic(dir, "config.json", cfg)) return pfail("Io", "cannot write " + dir + "/config.json");
  return GPRX_OK;
}

gprx_status persist_read(const std::string& dir, PersistModel& m, bool with_factor_data) {
  std::string text, err;
  if (!read_file(dir + "/config.json", text)) return pfail("Io", "cannot read " + dir + "/config.json");
  Json c;
  if (!parse_json(text, c, err) || c.kind != Json::OBJ) return pfail("Config", "config.json: " + err);
  const Json* fv = c.get("format_version");
  if (!fv || fv->kind != Json::NUM) return pfail("Config", "config.json has no format_version");
  if (fv->num != 1.0)
    return set_error(GPRX_UNSUPPORTED_PERSIST_VERSION,
                     "persist format_version " + fmt_num(fv->num) + " (this backend reads 1)");
  const Json* model = c.get("model");
  if (model && !(model->kind == Json::STR && model->str == "exact"))
    return pfail("WrongModel", "config.json holds a " + (model->kind == Json::STR ? model->str : std::string("?")) +
                                   " model; this loader reads exact models");
  if (c.get("distance")) return pfail("WrongModel", "a distance-kernel model; this loader reads coordinate models");
  auto str_or = [&](const char* k, const char* dflt) -> std::string {
    const Json* v = c.get(k);
    return v && v->kind == Json::STR ? v->str : std::string(dflt);
  };
  if (str_or("precision", "double") != "double")
    return pfail("Config", "precision '" + str_or("precision", "") + "' (this backend stores double)");
  if (str_or("math", "accurate") != "accurate") return pfail("Config", "math '" + str_or("math", "") + "'");
  for (const char* k : {"x_unfitted", "y_unfitted", "x_transform", "y_transform"}) {
    const Json* v = c.get(k);
    if (!v) return pfail("Config", std::string("config.json has no ") + k);
    if (!(v->kind == Json::STR && v->str == "identity"))
      return pfail("Config", std::string(k) + " is not the identity map (not supported by this backend)");
  }
  const Json* n = c.get("n");
  const Json* d = c.get("d");
  const Json* hf = c.get("has_factor");
  if (!n || n->kind != Json::NUM || !d || d->kind != Json::NUM || !hf || hf->kind != Json::BOOL)
    return pfail("Config", "config.json needs n, d and has_factor");
  if (n->num <= 0 || d->num <= 0) return set_error(GPRX_EMPTY_INPUT, "persist: n or d is 0");
  m.n = (long long)n->num;
  m.d = (long long)d->num;
  m.has_factor = hf->b;
  const std::string fk = str_or("factor_kind", "");
  if (fk != "llt" && fk != "ldlt") return pfail("Config", "factor_kind must be llt or ldlt");
  m.ldlt = fk == "ldlt";
  const Json* fj = c.get("factor_jitter");
  m.factor_jitter = fj && fj->kind == Json::NUM ? fj->num : 0.0;
  // kernel, likelihood, jitter
  const Json* k = c.get("kernel");
  if (!k) return pfail("Config", "config.json has no kernel");
  m.nodes.clear();
  m.theta.clear();
  if (!decode_kernel(*k, m.nodes, m.theta, err)) return pfail("Config", err);
  const Json* lik = c.get("likelihood");
  double noise = 0.0;
  if (!lik || !read_bounded(lik->get("noise_variance"), noise, err)) return pfail("Config", "likelihood: " + err);
  m.log_noise = std::log(noise);
  gprx_options_default(&m.jitter);
  const Json* j = c.get("jitter");
  if (!j || j->kind != Json::OBJ || j->obj.size() != 1) return pfail("Config", "jitter must be fixed or adaptive");
  const Json& jb = j->obj[0].second;
  if (j->obj[0].first == "fixed") {
    const Json* v = jb.get("jitter");
    if (!v || v->kind != Json::NUM || !(v->num >= 0.0) || !std::isfinite(v->num))
      return pfail("Config", "fixed jitter must be a finite number ≥ 0");
    m.jitter.jitter_kind = GPRX_JITTER_FIXED;
    m.jitter.jitter_initial = v->num;
  } else if (j->obj[0].first == "adaptive") {
    const Json* a = jb.get("initial");
    const Json* mu = jb.get("multiplier");
    const Json* r = jb.get("max_retries");
    const Json* mx = jb.get("max_jitter");
    if (!a || !mu || !r || !mx || a->kind != Json::NUM || mu->kind != Json::NUM || r->kind != Json::NUM ||
        mx->kind != Json::NUM || !(a->num > 0.0) || !(mu->num > 1.0) || r->num < 0 || !(mx->num >= a->num))
      return pfail("Config", "adaptive jitter needs initial > 0, multiplier > 1, max_retries ≥ 0, max_jitter ≥ initial");
    m.jitter.jitter_kind = GPRX_JITTER_ADAPTIVE;
    m.jitter.jitter_initial = a->num;
    m.jitter.jitter_multiplier = mu->num;
    m.jitter.jitter_max_retries = (int32_t)r->num;
    m.jitter.jitter_max = mx->num;
  } else {
    return pfail("Config", "jitter must be fixed or adaptive");
  }
  m.ids.clear();
  if (m.ldlt) {
    const Json* ids = c.get("point_ids");
    const Json* nx = c.get("next_point_id");
    if (!ids || ids->kind != Json::ARR || !nx || nx->kind != Json::NUM)
      return pfail("Config", "an ldlt model needs point_ids and next_point_id");
    if ((long long)ids->arr.size() != m.n) return pfail("Config", "point_ids has the wrong length");
    for (auto& e : ids->arr) m.ids.push_back((uint64_t)e.num);
    m.next_id = (uint64_t)nx->num;
  }
  // tensors
  auto mp = std::make_shared<Mapped>();
  std::map<std::string, TensorIn> ts;
  gprx_status st = map_safetensors(dir + "/model.safetensors", *mp, ts);
  if (st != GPRX_OK) return st;
  auto need = [&](const char* name, std::vector<long long> shape) -> const TensorIn* {
    auto it = ts.find(name);
    if (it == ts.end() || it->second.shape != shape) return nullptr;
    return &it->second;
  };
  const TensorIn* tx = need("x", {m.n, m.d});
  const TensorIn* ty = need("y", {m.n});
  if (!tx || !ty) return pfail("Tensor", "x [n, d] and y [n] are required");
  m.x.assign(tx->data, tx->data + tx->count);
  m.y.assign(ty->data, ty->data + ty->count);
  m.l_map = nullptr;
  m.alpha.clear();
  if (m.has_factor) {
    const TensorIn* tl = need("l", {m.n, m.n});
    const TensorIn* ta = need("alpha", {m.n});
    if (!tl || !ta) return pfail("Tensor", "has_factor needs l [n, n] and alpha [n]");
    m.alpha.assign(ta->data, ta->data + ta->count);
    if (with_factor_data) {
      m.l_map = tl->data;  // read straight from the mapping
      m.mapping = mp;
    }
  }
  return GPRX_OK;
}

}  // namespace gprx

using namespace gprx;

extern "C" {

gprx_status gprx_persist_inspect(const char* dir, gprx_persist_info* out) {
  if (!dir || !out) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  PersistModel m;
  gprx_status st = persist_read(dir, m, false);
  if (st != GPRX_OK) return st;
  out->n = (uint64_t)m.n;
  out->d = (uint64_t)m.d;
  out->n_nodes = (int32_t)m.nodes.size();
  out->n_theta = (int32_t)m.theta.size() + 1;
  out->has_factor = m.has_factor ? 1 : 0;
  out->factor_kind = m.ldlt ? 1 : 0;
  out->factor_jitter = m.factor_jitter;
  out->jitter = m.jitter;
  out->next_point_id = m.next_id;
  return GPRX_OK;
}

gprx_status gprx_persist_read(const char* dir, gprx_kernel_node* nodes, double* theta, double* x, double* y,
                              double* l, double* alpha, uint64_t* point_ids) {
  if (!dir || !nodes || !theta || !x || !y) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  PersistModel m;
  gprx_status st = persist_read(dir, m, l != nullptr);
  if (st != GPRX_OK) return st;
  std::copy(m.nodes.begin(), m.nodes.end(), nodes);
  std::copy(m.theta.begin(), m.theta.end(), theta);
  theta[m.theta.size()] = m.log_noise;
  std::copy(m.x.begin(), m.x.end(), x);
  std::copy(m.y.begin(), m.y.end(), y);
  if (m.has_factor && l) std::copy(m.l_map, m.l_map + (size_t)m.n * m.n, l);
  if (m.has_factor && alpha) std::copy(m.alpha.begin(), m.alpha.end(), alpha);
  if (m.ldlt && point_ids) std::copy(m.ids.begin(), m.ids.end(), point_ids);
  return GPRX_OK;
}

gprx_status gprx_persist_write(const char* dir, const double* x, uint64_t n, uint64_t d, const double* y,
                               const gprx_kernel_node* nodes, int32_t n_nodes, const double* theta, int32_t n_theta,
                               const gprx_options* jitter, const double* l, const double* alpha, int32_t factor_kind,
                               double factor_jitter, const uint64_t* point_ids, uint64_t next_point_id) {
  if (!dir || !x || !y || !nodes || !theta || n_theta < 1) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (factor_kind == 1 && !point_ids) return set_error(GPRX_INVALID_ARGUMENT, "an ldlt model needs point ids");
  PersistModel m;
  m.n = (long long)n;
  m.d = (long long)d;
  m.nodes.assign(nodes, nodes + n_nodes);
  m.theta.assign(theta, theta + n_theta - 1);
  m.log_noise = theta[n_theta - 1];
  if (jitter) m.jitter = *jitter;
  else gprx_options_default(&m.jitter);
  m.x.assign(x, x + n * d);
  m.y.assign(y, y + n);
  m.has_factor = l != nullptr && alpha != nullptr;
  m.ldlt = factor_kind == 1;
  m.factor_jitter = factor_jitter;
  if (m.has_factor) {
    m.l.assign(l, l + n * n);
    for (uint64_t j = 0; j < n; ++j)  // zero above the diagonal (the layout of l)
      for (uint64_t i = 0; i < j; ++i) m.l[i + j * n] = 0.0;
    m.alpha.assign(alpha, alpha + n);
  }
  if (point_ids) m.ids.assign(point_ids, point_ids + n);
  m.next_id = next_point_id;
  return persist_write(dir, m);
}

}  // extern "C"
