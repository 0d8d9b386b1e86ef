#include "param_files.h"

#include <sys/stat.h>

#include <algorithm>
#include <array>
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

#include "dftb_params.h"
#include "params.h"

namespace sgb {

// ---------------------------------------------------------------------------
// A small JSON reader (RFC 8259 values; numbers through std::from_chars, so
// every decimal literal becomes the correctly rounded double, independent of
// the process locale).
// ---------------------------------------------------------------------------
namespace {

struct Json {
  enum Kind { kNull, kBool, kNumber, kString, kArray, kObject } kind = kNull;
  double number = 0;
  bool boolean = false;
  std::string text;
  std::vector<Json> items;
  std::vector<std::pair<std::string, Json>> members;
  const Json* get(const char* key) const {
    for (const auto& kv : members)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
};

class JsonReader {
 public:
  explicit JsonReader(const std::string& s) : s_(s) {}
  bool parse(Json& out, std::string& err) {
    skip();
    if (!value(out, 0)) {
      err = error_;
      return false;
    }
    skip();
    if (p_ != s_.size()) {
      err = where("unexpected characters after the top-level value");
      return false;
    }
    return true;
  }

 private:
  const std::string& s_;
  size_t p_ = 0;
  std::string error_;

  std::string where(const std::string& what) const {
    int line = 1 + (int)std::count(s_.begin(), s_.begin() + std::min(p_, s_.size()), '\n');
    return what + " (line " + std::to_string(line) + ")";
  }
  bool fail(const std::string& what) {
    if (error_.empty()) error_ = where(what);
    return false;
  }
  void skip() {
    while (p_ < s_.size() && (s_[p_] == ' ' || s_[p_] == '\t' || s_[p_] == '\n' || s_[p_] == '\r')) ++p_;
  }
  bool literal(const char* w) {
    const size_t n = std::strlen(w);
    if (s_.compare(p_, n, w) != 0) return false;
    p_ += n;
    return true;
  }
  bool value(Json& v, int depth) {
    if (depth > 64) return fail("nesting too deep");
    if (p_ >= s_.size()) return fail("unexpected end of input");
    const char c = s_[p_];
    if (c == '{') return object(v, depth);
    if (c == '[') return array(v, depth);
    if (c == '"') {
      v.kind = Json::kString;
      return string(v.text);
    }
    if (c == '-' || (c >= '0' && c <= '9')) return number(v);
    if (literal("true")) {
      v.kind = Json::kBool;
      v.boolean = true;
      return true;
    }
    if (literal("false")) {
      v.kind = Json::kBool;
      return true;
    }
    if (literal("null")) {
      v.kind = Json::kNull;
      return true;
    }
    return fail("invalid value");
  }
  bool number(Json& v) {
    const char* b = s_.data() + p_;
    const char* e = s_.data() + s_.size();
    double x = 0;
    auto r = std::from_chars(b, e, x);
    if (r.ec != std::errc() || r.ptr == b) return fail("invalid number");
    v.kind = Json::kNumber;
    v.number = x;
    p_ += (size_t)(r.ptr - b);
    return true;
  }
  bool string(std::string& out) {
    ++p_;  // opening quote
    out.clear();
    while (p_ < s_.size()) {
      const char c = s_[p_++];
      if (c == '"') return true;
      if (c != '\\') {
        out.push_back(c);
        continue;
      }
      if (p_ >= s_.size()) break;
      const char esc = s_[p_++];
      switch (esc) {
        case '"': out.push_back('"'); break;
        case '\\': out.push_back('\\'); break;
        case '/': out.push_back('/'); break;
        case 'b': out.push_back('\b'); break;
        case 'f': out.push_back('\f'); break;
        case 'n': out.push_back('\n'); break;
        case 'r': out.push_back('\r'); break;
        case 't': out.push_back('\t'); break;
        case 'u': {
          if (p_ + 4 > s_.size()) return fail("truncated \\u escape");
          unsigned cp = 0;
          auto r = std::from_chars(s_.data() + p_, s_.data() + p_ + 4, cp, 16);
          if (r.ec != std::errc() || r.ptr != s_.data() + p_ + 4) return fail("invalid \\u escape");
          p_ += 4;
          if (cp < 0x80) {
            out.push_back((char)cp);
          } else if (cp < 0x800) {
            out.push_back((char)(0xC0 | (cp >> 6)));
            out.push_back((char)(0x80 | (cp & 0x3F)));
          } else {
            out.push_back((char)(0xE0 | (cp >> 12)));
            out.push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
            out.push_back((char)(0x80 | (cp & 0x3F)));
          }
          break;
        }
        default: return fail("invalid escape in string");
      }
    }
    return fail("unterminated string");
  }
  bool array(Json& v, int depth) {
    v.kind = Json::kArray;
    ++p_;
    skip();
    if (p_ < s_.size() && s_[p_] == ']') {
      ++p_;
      return true;
    }
    for (;;) {
      v.items.emplace_back();
      skip();
      if (!value(v.items.back(), depth + 1)) return false;
      skip();
      if (p_ < s_.size() && s_[p_] == ',') {
        ++p_;
        continue;
      }
      if (p_ < s_.size() && s_[p_] == ']') {
        ++p_;
        return true;
      }
      return fail("expected ',' or ']'");
    }
  }
  bool object(Json& v, int depth) {
    v.kind = Json::kObject;
    ++p_;
    skip();
    if (p_ < s_.size() && s_[p_] == '}') {
      ++p_;
      return true;
    }
    for (;;) {
      skip();
      if (p_ >= s_.size() || s_[p_] != '"') return fail("expected a member name");
      std::string key;
      if (!string(key)) return false;
      skip();
      if (p_ >= s_.size() || s_[p_] != ':') return fail("expected ':'");
      ++p_;
      skip();
      v.members.emplace_back(std::move(key), Json());
      if (!value(v.members.back().second, depth + 1)) return false;
      skip();
      if (p_ < s_.size() && s_[p_] == ',') {
        ++p_;
        continue;
      }
      if (p_ < s_.size() && s_[p_] == '}') {
        ++p_;
        return true;
      }
      return fail("expected ',' or '}'");
    }
  }
};

bool read_file(const std::string& path, std::string& text) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  std::ostringstream ss;
  ss << f.rdbuf();
  text = ss.str();
  return true;
}

// (modification time, size) of a regular file; false when it is not one
bool file_stamp(const std::string& path, std::pair<long long, long long>& stamp) {
  struct stat st;
  if (stat(path.c_str(), &st) != 0 || !S_ISREG(st.st_mode)) return false;
  stamp = {(long long)st.st_mtim.tv_sec * 1000000000LL + st.st_mtim.tv_nsec, (long long)st.st_size};
  return true;
}

// modification time of a directory (changes when entries are added, removed
// or replaced by rename); false when path is not a directory
bool directory_stamp(const std::string& path, long long& stamp) {
  struct stat st;
  if (stat(path.c_str(), &st) != 0 || !S_ISDIR(st.st_mode)) return false;
  stamp = (long long)st.st_mtim.tv_sec * 1000000000LL + st.st_mtim.tv_nsec;
  return true;
}

}  // namespace

// ---------------------------------------------------------------------------
// NDDO parameters.json
// ---------------------------------------------------------------------------
const NddoRawAtomic* NddoParamSet::find(int Z) const {
  for (const auto& a : atomic)
    if (a.Z == Z) return &a;
  return nullptr;
}

const NddoRawDiatomic* NddoParamSet::find_pair(int z1, int z2) const {
  for (const auto& d : diatomic)
    if ((d.z1 == z1 && d.z2 == z2) || (d.z1 == z2 && d.z2 == z1)) return &d;
  return nullptr;
}

bool sto6g_expansion(int n, int l, double zeta, double* exp6, double* coef6) {
  if (l < 0 || l > 1 || !(zeta > 0)) return false;
  // a donor: any embedded element whose shell (n, l) carries an expansion
  for (Method m : {kPM6, kAM1, kMNDO}) {
    size_t count = 0;
    const NddoRawAtomic* tab = nddo_embedded_atomic(m, count);
    for (size_t i = 0; i < count; ++i) {
      const NddoRawAtomic& r = tab[i];
      const double z0 = r.v[l == 0 ? kRawZetaS : kRawZetaP];
      const double* e0 = l == 0 ? r.s_exp : r.p_exp;
      const double* c0 = l == 0 ? r.s_coef : r.p_coef;
      if (nddo_shell_n(r.Z, l) != n || !(z0 > 0) || e0[0] == 0.0) continue;
      if (l == 1 && r.Z == 1) continue;
      const double s = zeta / z0;
      const double fe = s * s;
      const double fc = l == 0 ? s * std::sqrt(s) : s * s * std::sqrt(s);
      for (int k = 0; k < 6; ++k) {
        exp6[k] = e0[k] * fe;
        coef6[k] = c0[k] * fc;
      }
      return true;
    }
  }
  return false;
}

namespace {

bool number_at(const Json* obj, const char* key, double& out, std::string& err, const std::string& where) {
  const Json* v = obj ? obj->get(key) : nullptr;
  if (!v || v->kind != Json::kNumber) {
    err = where + ": missing number '" + key + "'";
    return false;
  }
  out = v->number;
  return true;
}

bool spd_at(const Json* pack, const char* key, double* spd, std::string& err, const std::string& where) {
  const Json* o = pack->get(key);
  if (!o || o->kind != Json::kObject) {
    err = where + ": missing object '" + key + "'";
    return false;
  }
  const std::string w = where + "." + key;
  return number_at(o, "s", spd[0], err, w) && number_at(o, "p", spd[1], err, w) && number_at(o, "d", spd[2], err, w);
}

bool integer_value(const Json* v, int& out) {
  if (!v || v->kind != Json::kNumber || v->number != std::floor(v->number) || v->number < 1 || v->number > 118)
    return false;
  out = (int)v->number;
  return true;
}

// One "atomic" entry: {"key": Z, "value": {"pack": {...}, "gaussianRepulsion": [...]}}
bool atomic_record(Method m, const Json& entry, NddoRawAtomic& r, std::string& err) {
  int Z = 0;
  if (entry.kind != Json::kObject || !integer_value(entry.get("key"), Z)) {
    err = "atomic entry without an integer 'key' (atomic number)";
    return false;
  }
  const std::string where = "atomic[Z=" + std::to_string(Z) + "]";
  const Json* value = entry.get("value");
  const Json* pack = value ? value->get("pack") : nullptr;
  if (!pack || pack->kind != Json::kObject) {
    err = where + ": missing 'value.pack'";
    return false;
  }
  double u[3], beta[3], zeta[3];
  std::memset(&r, 0, sizeof(r));
  r.Z = Z;
  if (!spd_at(pack, "oneCenterEnergy", u, err, where) || !spd_at(pack, "beta", beta, err, where) ||
      !spd_at(pack, "orbitalExponent", zeta, err, where))
    return false;
  r.v[kRawUss] = u[0];
  r.v[kRawUpp] = u[1];
  r.v[kRawBetaS] = beta[0];
  r.v[kRawBetaP] = beta[1];
  r.v[kRawZetaS] = zeta[0];
  r.v[kRawZetaP] = zeta[1];
  r.has_d = (u[2] != 0 || zeta[2] != 0) ? 1 : 0;
  static const struct { const char* key; int index; } scalars[] = {
      {"gss", kRawGss}, {"gpp", kRawGpp}, {"gsp", kRawGsp},     {"gp2", kRawGp2},
      {"hsp", kRawHsp}, {"pcore", kRawPcore}, {"alpha", kRawAlpha}};
  for (const auto& s : scalars)
    if (!number_at(pack, s.key, r.v[s.index], err, where + ".pack")) return false;
  const Json* gauss = value->get("gaussianRepulsion");
  if (gauss && gauss->kind != Json::kArray) {
    err = where + ": 'gaussianRepulsion' is not an array";
    return false;
  }
  if (gauss) {
    if (gauss->items.size() > 4) {
      err = where + ": more than four Gaussian core-repulsion terms";
      return false;
    }
    r.n_gauss = (int)gauss->items.size();
    for (int k = 0; k < r.n_gauss; ++k) {
      const Json& g = gauss->items[k];
      const std::string w = where + ".gaussianRepulsion[" + std::to_string(k) + "]";
      if (!number_at(&g, "a", r.ga[k], err, w) || !number_at(&g, "b", r.gb[k], err, w) ||
          !number_at(&g, "c", r.gc[k], err, w))
        return false;
    }
  }
  // STO-6G shells: the embedded expansion where the exponent is the embedded
  // one (bit-identical to the built-in set), else the scaled expansion
  size_t count = 0;
  const NddoRawAtomic* tab = nddo_embedded_atomic(m, count);
  const NddoRawAtomic* own = nullptr;
  for (size_t i = 0; i < count; ++i)
    if (tab[i].Z == Z) own = &tab[i];
  for (int l = 0; l < 2; ++l) {
    const double z = l == 0 ? zeta[0] : zeta[1];
    double* e = l == 0 ? r.s_exp : r.p_exp;
    double* c = l == 0 ? r.s_coef : r.p_coef;
    if (l == 1 && (Z == 1 || z == 0)) continue;  // no p shell
    if (own && own->v[l == 0 ? kRawZetaS : kRawZetaP] == z) {
      std::memcpy(e, l == 0 ? own->s_exp : own->p_exp, 6 * sizeof(double));
      std::memcpy(c, l == 0 ? own->s_coef : own->p_coef, 6 * sizeof(double));
    } else if (!sto6g_expansion(nddo_shell_n(Z, l), l, z, e, c)) {
      err = where + ": no STO-6G expansion for the " + (l == 0 ? "s" : "p") + " shell (exponent " +
            std::to_string(z) + ")";
      return false;
    }
  }
  return true;
}

bool parse_nddo_json(Method m, const std::string& text, NddoParamSet& set, std::string& err) {
  Json root;
  if (!JsonReader(text).parse(root, err)) return false;
  const Json* atomic = root.kind == Json::kObject ? root.get("atomic") : nullptr;
  if (!atomic || atomic->kind != Json::kArray) {
    err = "no 'atomic' array";
    return false;
  }
  for (const Json& entry : atomic->items) {
    NddoRawAtomic r;
    if (!atomic_record(m, entry, r, err)) return false;
    if (set.find(r.Z)) {
      err = "element Z=" + std::to_string(r.Z) + " appears twice in 'atomic'";
      return false;
    }
    set.atomic.push_back(r);
  }
  const Json* diatomic = root.get("diatomic");
  if (diatomic && diatomic->kind != Json::kArray && diatomic->kind != Json::kNull) {
    err = "'diatomic' is not an array";
    return false;
  }
  if (diatomic && diatomic->kind == Json::kArray)
    for (const Json& entry : diatomic->items) {
      const Json* key = entry.kind == Json::kObject ? entry.get("key") : nullptr;
      NddoRawDiatomic d{};
      if (!key || !integer_value(key->get("first"), d.z1) || !integer_value(key->get("second"), d.z2)) {
        err = "diatomic entry without integer 'key.first' / 'key.second'";
        return false;
      }
      const std::string w = "diatomic[" + std::to_string(d.z1) + "," + std::to_string(d.z2) + "]";
      const Json* value = entry.get("value");
      if (!number_at(value, "exponent", d.exponent, err, w) || !number_at(value, "factor", d.factor, err, w))
        return false;
      set.diatomic.push_back(d);
    }
  return true;
}

struct NddoCacheEntry {
  std::pair<long long, long long> stamp;
  std::shared_ptr<const NddoParamSet> set;
};

}  // namespace

std::shared_ptr<const NddoParamSet> nddo_parameter_set(Method m, const std::string& path, std::string& err) {
  static std::mutex mu;
  static std::map<std::pair<int, std::string>, NddoCacheEntry> cache;
  if (is_dftb(m)) {
    err = "NDDO parameter files apply to MNDO, AM1 and PM6 only";
    return nullptr;
  }
  std::pair<long long, long long> stamp{0, 0};
  if (!path.empty() && !file_stamp(path, stamp)) {
    err = "parameter file to read does not exist: '" + path + "'";
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find({(int)m, path});
  if (it != cache.end() && it->second.stamp == stamp) return it->second.set;
  auto set = std::make_shared<NddoParamSet>();
  set->source = path;
  if (path.empty()) {
    size_t n = 0, nd = 0;
    const NddoRawAtomic* a = nddo_embedded_atomic(m, n);
    const NddoRawDiatomic* d = nddo_embedded_diatomic(m, nd);
    set->atomic.assign(a, a + n);
    set->diatomic.assign(d, d + nd);
  } else {
    std::string text;
    if (!read_file(path, text)) {
      err = "parameter file cannot be opened: '" + path + "'";
      return nullptr;
    }
    std::string why;
    if (!parse_nddo_json(m, text, *set, why)) {
      err = "parameter file '" + path + "': " + why;
      return nullptr;
    }
  }
  cache[{(int)m, path}] = NddoCacheEntry{stamp, set};
  return set;
}

// ---------------------------------------------------------------------------
// DFTB Slater-Koster directories
// ---------------------------------------------------------------------------
const DftbElemRaw* DftbSetData::find_elem(int Z) const {
  for (const auto& e : elems)
    if (e.Z == Z) return &e;
  return nullptr;
}

const DftbPairRaw* DftbSetData::find_pair(int z1, int z2) const {
  for (const auto& p : pairs)
    if (p.z1 == z1 && p.z2 == z2) return &p;
  return nullptr;
}

namespace {

// the s/p elements of the DFTB engine
const char* const kSymbols[] = {"", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne"};
constexpr int kMaxSpZ = 10;
// kept columns of the 20 (Hdd0 Hdd1 Hdd2 Hpd0 Hpd1 Hpp0 Hpp1 Hsd0 Hsp0 Hss0, then the overlaps)
constexpr int kKeep[8] = {19, 9, 18, 8, 15, 5, 16, 6};

bool parse_double(const std::string& t, double& x) {
  std::string s = t;
  for (char& c : s)
    if (c == 'd' || c == 'D') c = 'e';  // Fortran exponents
  const char* b = s.data();
  const char* e = b + s.size();
  if (*b == '+') ++b;
  auto r = std::from_chars(b, e, x);
  return r.ec == std::errc() && r.ptr == e;
}

// The numbers of one line (blank- or comma-separated, "n*v" = n copies of v);
// false when a token is not a number.  plain counts tokens without '*'.
bool line_numbers(const std::string& line, std::vector<double>& out, int* plain = nullptr) {
  out.clear();
  int np = 0;
  size_t i = 0;
  while (i < line.size()) {
    while (i < line.size() && (line[i] == ' ' || line[i] == '\t' || line[i] == ',' || line[i] == '\r')) ++i;
    if (i >= line.size()) break;
    size_t j = i;
    while (j < line.size() && line[j] != ' ' && line[j] != '\t' && line[j] != ',' && line[j] != '\r') ++j;
    const std::string tok = line.substr(i, j - i);
    const size_t star = tok.find('*');
    double x;
    if (star != std::string::npos) {
      unsigned n = 0;
      auto r = std::from_chars(tok.data(), tok.data() + star, n);
      if (r.ec != std::errc() || r.ptr != tok.data() + star || !parse_double(tok.substr(star + 1), x)) return false;
      out.insert(out.end(), n, x);
    } else {
      if (!parse_double(tok, x)) return false;
      out.push_back(x);
      ++np;
    }
    i = j;
  }
  if (plain) *plain = np;
  return true;
}

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

struct SkfFile {
  double grid = 0;
  bool has_atomic = false;
  double atomic[10] = {};  // Ed Ep Es SPE Ud Up Us fd fp fs
  std::vector<std::array<double, 8>> rows;
  int n_spline_header = 0;
  double cutoff = 0, a1 = 0, a2 = 0, a3 = 0, c4 = 0, c5 = 0;
  std::vector<DftbSplineRaw> splines;
};

// One .skf file, following forwarding files ("X-Y.skf" as the whole content)
bool read_skf(const std::string& dir, std::string path, SkfFile& f, std::string& err) {
  std::string text;
  for (int hop = 0;; ++hop) {
    if (!read_file(path, text)) {
      err = "cannot open '" + path + "'";
      return false;
    }
    const std::string t = trim(text);
    const bool forward = t.size() > 4 && t.compare(t.size() - 4, 4, ".skf") == 0 &&
                         std::all_of(t.begin(), t.end() - 4, [](char c) { return std::isalpha((unsigned char)c) || c == '-'; });
    if (!forward) break;
    if (hop >= 16) {
      err = "SKF forwarding does not end at '" + path + "'";
      return false;
    }
    path = dir + "/" + t;
    std::pair<long long, long long> st;
    if (!file_stamp(path, st)) {
      err = "SKF forwarding could not be resolved: '" + path + "'";
      return false;
    }
  }
  std::vector<std::string> lines;
  {
    std::istringstream ss(text);
    std::string l;
    while (std::getline(ss, l)) lines.push_back(l);
  }
  auto bad = [&](size_t k, const char* what) {
    err = "'" + path + "' line " + std::to_string(k + 1) + ": " + what;
    return false;
  };
  std::vector<double> v;
  size_t k = 0;
  if (lines.empty() || !line_numbers(lines[0], v) || v.size() < 2) return bad(0, "expected grid distance and count");
  f.grid = v[0];
  k = 1;
  int plain = 0;
  // optional line of exactly ten numbers: the atomic parameters
  if (k < lines.size() && line_numbers(lines[k], v, &plain) && v.size() == 10 && plain == 10) {
    f.has_atomic = true;
    std::copy(v.begin(), v.end(), f.atomic);
    ++k;
  }
  if (k >= lines.size() || !line_numbers(lines[k], v) || v.empty()) return bad(k, "expected the mass / polynomial line");
  ++k;
  // integral table: numeric lines up to the first other line
  for (; k < lines.size(); ++k) {
    if (trim(lines[k]).empty() || !line_numbers(lines[k], v) || v.empty()) break;
    if (v.size() < 20) return bad(k, "integral line with fewer than 20 numbers");
    std::array<double, 8> row;
    for (int c = 0; c < 8; ++c) row[c] = v[kKeep[c]];
    f.rows.push_back(row);
  }
  while (k < lines.size() && trim(lines[k]).empty()) ++k;
  if (k >= lines.size() || trim(lines[k]).rfind("Spline", 0) != 0) return bad(k, "expected the 'Spline' block");
  ++k;
  while (k < lines.size() && trim(lines[k]).empty()) ++k;
  if (k >= lines.size() || !line_numbers(lines[k], v) || v.size() < 2) return bad(k, "expected spline count and cutoff");
  f.n_spline_header = (int)v[0];
  f.cutoff = v[1];
  ++k;
  if (k >= lines.size() || !line_numbers(lines[k], v) || v.size() < 3) return bad(k, "expected a1 a2 a3");
  f.a1 = v[0];
  f.a2 = v[1];
  f.a3 = v[2];
  ++k;
  for (; k < lines.size(); ++k) {
    if (!line_numbers(lines[k], v) || v.size() < 6) break;
    f.splines.push_back(DftbSplineRaw{v[0], v[1], v[2], v[3], v[4], v[5]});
    if (v.size() >= 8) {
      f.c4 = v[6];
      f.c5 = v[7];
    }
  }
  if (f.rows.empty()) return bad(k, "no integral table");
  if (f.splines.empty()) return bad(k, "no repulsion spline");
  return true;
}

// X-Y.skf, then XY.skf, each as given and in lower case (ParameterSet.cpp:34-66)
bool find_skf(const std::string& dir, int za, int zb, std::string& path) {
  const std::string a = kSymbols[za], b = kSymbols[zb];
  for (const std::string& name : {a + "-" + b + ".skf", a + b + ".skf"}) {
    std::string lower = name;
    std::transform(lower.begin(), lower.end(), lower.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    for (const std::string& n : {name, lower}) {
      std::pair<long long, long long> st;
      if (file_stamp(dir + "/" + n, st)) {
        path = dir + "/" + n;
        return true;
      }
    }
  }
  return false;
}

int symbol_to_z(const std::string& s) {
  for (int z = 1; z <= kMaxSpZ; ++z)
    if (s == kSymbols[z]) return z;
  return 0;
}

bool load_skf_directory(const std::string& dir, DftbSetData& set, std::string& err) {
  set.name = dir;
  // Hubbard derivatives and spin constants (SkfParser.cpp:255-330)
  std::map<int, double> hubbard;
  std::map<int, std::array<double, 4>> spin;  // W_ss, W_sp, W_ps, W_pp
  std::string text;
  if (read_file(dir + "/hubbard.dat", text)) {
    std::istringstream ss(text);
    std::string sym, val;
    while (ss >> sym >> val) {
      double x;
      if (!parse_double(val, x)) {
        err = "hubbard.dat: '" + val + "' is not a number";
        return false;
      }
      if (int z = symbol_to_z(sym)) hubbard[z] = x;
    }
  }
  if (read_file(dir + "/spin.dat", text)) {
    std::istringstream ss(text);
    std::string line;
    while (std::getline(ss, line)) {
      if (line.find('#') != std::string::npos) continue;
      std::istringstream ls(line);
      std::string sym;
      double w[9];
      if (!(ls >> sym)) continue;
      int n = 0;
      while (n < 9 && (ls >> w[n])) ++n;
      if (n < 9) {
        err = "spin.dat: expected nine constants for '" + sym + "'";
        return false;
      }
      // order W00 W01 W10 W11 W02 W12 W22 W20 W21: s-s and p-p are the first and fourth
      if (int z = symbol_to_z(sym)) spin[z] = {w[0], w[1], w[2], w[3]};
    }
  }
  // elements: those with a homonuclear file carrying atomic parameters
  std::vector<int> zs;
  for (int z = 1; z <= kMaxSpZ; ++z) {
    std::string path;
    if (!find_skf(dir, z, z, path)) continue;
    SkfFile f;
    if (!read_skf(dir, path, f, err)) return false;
    if (!f.has_atomic) {
      err = "'" + path + "' has no atomic parameter line";
      return false;
    }
    DftbElemRaw e{};
    e.Z = z;
    e.ed = f.atomic[0];
    e.ep = f.atomic[1];
    e.es = f.atomic[2];
    e.ud = f.atomic[4];
    e.up = f.atomic[5];
    e.us = f.atomic[6];
    // occupations are read as unsigned integers (SkfParser.cpp:157-167)
    e.fd = (double)(unsigned)f.atomic[7];
    e.fp = (double)(unsigned)f.atomic[8];
    e.fs = (double)(unsigned)f.atomic[9];
    auto h = hubbard.find(z);
    e.has_hubbard_derivative = h != hubbard.end();
    e.hubbard_derivative = e.has_hubbard_derivative ? h->second : 0.0;
    auto s = spin.find(z);
    e.has_spin = s != spin.end();
    e.wss = e.has_spin ? s->second[0] : 0.0;
    e.wsp = e.has_spin ? s->second[1] : 0.0;
    e.wps = e.has_spin ? s->second[2] : 0.0;
    e.wpp = e.has_spin ? s->second[3] : 0.0;
    set.elems.push_back(e);
    zs.push_back(z);
  }
  if (zs.empty()) {
    err = "no homonuclear Slater-Koster file of an s/p element (H to Ne) in '" + dir + "'";
    return false;
  }
  for (int za : zs)
    for (int zb : zs) {
      std::string path;
      if (!find_skf(dir, za, zb, path)) continue;  // reported when a molecule needs the pair
      SkfFile f;
      if (!read_skf(dir, path, f, err)) return false;
      DftbPairRaw p{};
      p.z1 = za;
      p.z2 = zb;
      p.grid = f.grid;
      p.rows = (int)f.rows.size();
      p.row0 = (int)(set.table.size() / 8);
      for (const auto& r : f.rows) set.table.insert(set.table.end(), r.begin(), r.end());
      p.n_spline = (int)f.splines.size();
      p.cutoff = f.cutoff;
      p.a1 = f.a1;
      p.a2 = f.a2;
      p.a3 = f.a3;
      p.c4 = f.c4;
      p.c5 = f.c5;
      p.spline0 = (int)set.splines.size();
      set.splines.insert(set.splines.end(), f.splines.begin(), f.splines.end());
      set.pairs.push_back(p);
    }
  return true;
}

}  // namespace

std::shared_ptr<const DftbSetData> dftb_parameter_set(const std::string& name, std::string& err) {
  if (auto s = dftb_embedded_set(name)) return s;
  long long stamp = 0;
  if (!directory_stamp(name, stamp)) {
    err = "no embedded DFTB parameters named '" + name + "' (mio-1-1, 3ob-3-1, 3ob-2-1) and no such directory";
    return nullptr;
  }
  static std::mutex mu;
  static std::map<std::string, std::pair<long long, std::shared_ptr<const DftbSetData>>> cache;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(name);
  if (it != cache.end() && it->second.first == stamp) return it->second.second;
  auto set = std::make_shared<DftbSetData>();
  std::string why;
  if (!load_skf_directory(name, *set, why)) {
    err = "DFTB parameter directory '" + name + "': " + why;
    return nullptr;
  }
  cache[name] = {stamp, set};
  return set;
}

}  // namespace sgb
