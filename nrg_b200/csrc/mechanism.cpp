// Mechanism / thermo / molar-mass deck reader.
//
// Semantics follow the reference readers (chemical_properties_class.f90:
// 222-451 reaction records, 453-635 reaction strings, 685-768 species block;
// thermophysical_properties_class.f90:1226-1311 NASA-7 records, 1313-1341
// molar masses).  The decks are read with Fortran list-directed rules, which
// this file models with a record cursor (Deck) and a value scanner:
//   * an item read skips blank records and returns the first value; values are
//     separated by blanks or commas, a slash ends the read, quotes delimit;
//   * "backspace" returns to the record the previous item read came from;
//   * reals may drop the exponent letter ("4.8749+04" == 4.8749e4).
#include "mechanism.hpp"

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace nrg {
namespace {

// ------------------------------------------------------------ records
class Deck {
 public:
  bool open(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return false;
    std::string line;
    while (std::getline(in, line)) {
      if (!line.empty() && line.back() == '\r') line.pop_back();
      recs_.push_back(line);
    }
    return true;
  }
  void rewind() { cur_ = 0; }
  void backspace() { if (cur_ > 0) --cur_; }
  bool eof() const { return cur_ >= recs_.size(); }
  const std::string& take() { return recs_[cur_++]; }
  size_t pos() const { return cur_; }
  void seek(size_t p) { cur_ = p; }
  const std::string& at(size_t i) const { return recs_[i]; }
  size_t size() const { return recs_.size(); }

  // List-directed read of `count` values starting at the next record.
  // Returns false on end of file before the first value.
  bool items(std::vector<std::string>* out, int count) {
    out->clear();
    const std::string* rec = nullptr;
    size_t i = 0;
    while ((int)out->size() < count) {
      if (!rec) {
        if (eof()) return !out->empty();
        rec = &take();
        i = 0;
      }
      while (i < rec->size() && ((*rec)[i] == ' ' || (*rec)[i] == '\t' || (*rec)[i] == ',')) ++i;
      if (i >= rec->size()) { rec = nullptr; continue; }
      char c = (*rec)[i];
      if (c == '/') return true;
      std::string v;
      if (c == '\'' || c == '"') {
        ++i;
        while (i < rec->size()) {
          if ((*rec)[i] == c) {
            if (i + 1 < rec->size() && (*rec)[i + 1] == c) { v += c; i += 2; continue; }
            ++i;
            break;
          }
          v += (*rec)[i++];
        }
      } else {
        while (i < rec->size() && (*rec)[i] != ' ' && (*rec)[i] != '\t' && (*rec)[i] != ',' &&
               (*rec)[i] != '/')
          v += (*rec)[i++];
      }
      out->push_back(v);
    }
    return true;
  }
  bool item(std::string* s) {
    std::vector<std::string> v;
    if (!items(&v, 1) || v.empty()) return false;
    *s = v[0];
    return true;
  }

 private:
  std::vector<std::string> recs_;
  size_t cur_ = 0;
};

std::string rtrim(std::string s) {
  while (!s.empty() && s.back() == ' ') s.pop_back();
  return s;
}
std::string ltrim(std::string s) {
  size_t i = 0;
  while (i < s.size() && s[i] == ' ') ++i;
  return s.substr(i);
}
bool same(const std::string& a, const std::string& b) { return rtrim(a) == rtrim(b); }

// Fortran real literal -> double (exponent letter optional before a sign).
bool fortran_real(const std::string& tok, double* out) {
  std::string t = ltrim(rtrim(tok)), norm;
  size_t i = 0;
  if (i < t.size() && (t[i] == '+' || t[i] == '-')) norm += t[i++];
  int digits = 0;
  while (i < t.size() && (std::isdigit((unsigned char)t[i]) || t[i] == '.')) {
    if (t[i] != '.') ++digits;
    norm += t[i++];
  }
  if (!digits) return false;
  if (i < t.size()) {
    char c = (char)std::toupper((unsigned char)t[i]);
    if (c == 'E' || c == 'D' || c == 'Q') ++i;
    else if (c != '+' && c != '-') return false;
    norm += 'E';
    if (i < t.size() && (t[i] == '+' || t[i] == '-')) norm += t[i++];
    if (i >= t.size() || !std::isdigit((unsigned char)t[i])) return false;
    while (i < t.size() && std::isdigit((unsigned char)t[i])) norm += t[i++];
  }
  if (i != t.size()) return false;
  *out = std::strtod(norm.c_str(), nullptr);
  return true;
}

// ------------------------------------------------------------ species
int species_index(const Mechanism& m, const std::string& name) {
  for (int i = 0; i < m.n(); ++i)
    if (same(name, m.species[i])) return i + 1;
  if (same(name, "M")) return m.n() + 1;
  return 0;
}

bool seek_keyword(Deck& d, const char* kw) {
  d.rewind();
  std::string s;
  while (d.item(&s))
    if (same(s, kw)) return true;
  return false;
}

// The species block is scanned one character at a time (non-advancing
// reads); a name ends at the first blank after a non-blank character, and an
// end of record reads as a blank.
bool read_species(Deck& d, Mechanism* m) {
  if (!seek_keyword(d, "SPECIES")) return false;
  size_t rec = d.pos(), col = 0;
  for (;;) {
    std::string acc = "  ";
    char letter = 'x';
    while (letter != ' ' || acc[acc.size() - 2] == ' ') {
      if (rec >= d.size()) return false;
      const std::string& line = d.at(rec);
      if (col < line.size()) {
        letter = line[col++];
      } else {
        letter = ' ';
        ++rec;
        col = 0;
      }
      acc += letter;
      if (acc.size() > 150) return false;
    }
    std::string name = rtrim(ltrim(acc));
    if (name == "END") break;
    m->species.push_back(name.substr(0, 20));
  }
  return !m->species.empty();
}

// ------------------------------------------------------------ reactions
struct Side {
  int idx[3] = {0, 0, 0};
  int count = 0;
};

// One side of a reaction string: "a", "2a", "a+b", "2a+b", "a+2b", "a+b+c".
void parse_side(const Mechanism& m, const std::string& s, Side* out, bool* unknown) {
  auto look = [&](const std::string& name) {
    int k = species_index(m, name);
    if (k == 0) *unknown = true;
    return k;
  };
  size_t p = s.find('+');
  if (p == std::string::npos) {
    if (!s.empty() && s[0] == '2') {
      out->idx[0] = out->idx[1] = look(s.substr(1));
      out->count = 2;
    } else {
      out->idx[0] = look(s);
      out->count = 1;
    }
    return;
  }
  std::string first = s.substr(0, p), rest = s.substr(p + 1);
  bool doubled = !first.empty() && first[0] == '2';
  if (doubled) {
    out->idx[0] = out->idx[1] = look(first.substr(1));
    out->count = 2;
  } else {
    out->idx[0] = look(first);
    out->count = 1;
  }
  size_t q = rest.find('+');
  if (q == std::string::npos) {
    if (!rest.empty() && rest[0] == '2') {
      out->idx[1] = out->idx[2] = look(rest.substr(1));
      out->count = 3;
    } else if (doubled) {
      out->idx[2] = look(rest);
      out->count = 3;
    } else {
      out->idx[1] = look(rest);
      out->count = 2;
    }
  } else {
    out->idx[1] = look(rest.substr(0, q));
    out->idx[2] = look(rest.substr(q + 1));
    out->count = 3;
  }
}

// Reaction record head, e.g. "H+O2(+M)<=>HO2(+M)".  Returns the arrow kind
// (0 none, 1 "=", 2 "=>", 3 "<=") and the two sides.
int split_reaction(const Mechanism& m, std::string s, Side* L, Side* R, bool* unknown,
                   bool* falloff) {
  size_t fo = s.find("(+M)");
  *falloff = fo != std::string::npos;
  if (*falloff) {
    // keep text before the first "(+M)" and drop the trailing "(+M)"
    size_t tail_end = s.size() >= 4 ? s.size() - 4 : 0;
    std::string mid = (fo + 4 < tail_end) ? s.substr(fo + 4, tail_end - (fo + 4)) : "";
    s = s.substr(0, fo) + mid;
  }
  int kind = 0;
  if (s.find('=') != std::string::npos) kind = 1;
  if (s.find("=>") != std::string::npos) kind = 2;
  if (s.find("<=") != std::string::npos) kind = 3;
  if (kind == 0) return 0;
  const char* arrow = kind == 1 ? "=" : (kind == 2 ? "=>" : "<=");
  size_t p = s.find(arrow);
  size_t skip = kind == 1 ? 1 : (kind == 2 ? 2 : 3);
  std::string left = s.substr(0, p);
  std::string right = p + skip <= s.size() ? s.substr(p + skip) : "";
  left = rtrim(left.substr(0, 20));   // character(len=20) holders
  right = rtrim(right.substr(0, 20));
  *unknown = false;
  parse_side(m, left, L, unknown);
  parse_side(m, right, R, unknown);
  return kind;
}

std::string read_reactions(Deck& d, double eff_default, Mechanism* m) {
  if (!seek_keyword(d, "REACTIONS")) return "REACTIONS keyword not found";
  bool enhanced = false;  // the reference never clears this flag
  int err = 0;
  std::string head;
  const int n = m->n();
  while (d.item(&head)) {
    if (head.size() > 150) head.resize(150);
    bool third_body = head.find("+M") != std::string::npos;
    Side L, R;
    bool unknown = false, falloff = false;
    int kind = split_reaction(*m, head, &L, &R, &unknown, &falloff);
    if (falloff) enhanced = true;
    if (kind == 0 || unknown) continue;
    Reaction rx;
    if (kind == 2) rx.type = third_body ? 6 : 5;
    else rx.type = third_body ? 1 : 0;
    if (third_body) enhanced = true;
    rx.n_left = L.count;
    rx.n_right = R.count;
    for (int i = 0; i < 3; ++i) { rx.left[i] = L.idx[i]; rx.right[i] = R.idx[i]; }

    std::vector<std::string> v;
    auto reals = [&](int k, double* dst) {
      d.backspace();
      err = 0;
      if (!d.items(&v, 1 + k) || (int)v.size() < 1 + k) { err = -1; return; }
      for (int i = 0; i < k; ++i)
        if (!fortran_real(v[1 + i], &dst[i])) { err = 1; return; }
    };
    double abe[3] = {0, 0, 0};
    reals(3, abe);
    rx.A = abe[0]; rx.beta = abe[1]; rx.E = abe[2];

    if (falloff) {
      std::string s;
      err = d.item(&s) ? 0 : -1;
      if (err == 0 && same(s, "LOW")) {
        rx.type = kind == 2 ? 7 : 2;
        double low[3] = {0, 0, 0};
        reals(3, low);
        rx.A_low = low[0]; rx.beta_low = low[1]; rx.E_low = low[2];
      }
      err = d.item(&s) ? 0 : -1;
      if (err == 0 && same(s, "TROE")) {
        rx.type = kind == 2 ? 7 : 3;
        reals(4, rx.troe);
      } else {
        d.backspace();
      }
    }
    m->reactions.push_back(rx);
    int r = m->r() - 1;
    m->eff.resize((size_t)m->r() * n, eff_default);

    if (err == 0) {
      std::string s;
      bool got = d.item(&s);
      if (got && s.find('/') != std::string::npos && enhanced) {
        // "NAME/value/ NAME/value/ ..." -- names not in the mechanism skipped
        std::string rest = s.substr(0, 150);
        while (!rtrim(rest).empty()) {
          size_t a = rest.find('/');
          if (a == std::string::npos) break;
          std::string name = rtrim(ltrim(rest.substr(0, a)));
          rest = rest.substr(a + 1);
          size_t b = rest.find('/');
          int k = species_index(*m, name);
          if (k > 0 && k <= n && b != std::string::npos) {
            double val;
            if (fortran_real(rest.substr(0, b), &val)) m->eff[(size_t)r * n + (k - 1)] = val;
          }
          if (b == std::string::npos) break;
          rest = rest.substr(b + 1);
        }
      } else if (got) {
        d.backspace();
      }
    }
  }
  return "";
}

// ------------------------------------------------------------ thermo
// NASA-7 records: numbers are cut at a class change from the set
// "-+E0123456789." (a '-' not following 'E' starts a new number); the
// record-number tokens (5th and 11th items) are skipped and reading stops
// after 14 coefficients -- the high-range set first, then the low-range set.
bool nasa7(Deck& d, const std::string& name, double a[2][7]) {
  for (int s = 0; s < 2; ++s)
    for (int i = 0; i < 7; ++i) a[s][i] = 0.0;
  d.rewind();
  std::string s;
  bool found = false;
  static const std::string cls = "-+E0123456789.";
  while (d.item(&s)) {
    if (s.size() > 100) s.resize(100);
    if (same(s, "END")) break;
    if (!same(s, name)) continue;
    found = true;
    int num = 0, i1 = 1, set = 2;
    while (num < 16) {
      if (d.eof()) return false;
      std::string line = rtrim(d.take().substr(0, 100));
      int prev = -1, begin = 1, len = (int)line.size();
      for (int i = 1; i <= len; ++i) {
        size_t f = cls.find(line[i - 1]);
        int cl = f == std::string::npos ? 0 : (int)f + 1;
        bool cut = (cl == 0 && prev > 0) || (cl == 1 && prev != 3 && prev > 0) ||
                   (cl != 0 && i == len);
        if (cut) {
          if (num == 5 || num == 11) {
            ++num;
          } else if (num == 16) {
            break;
          } else {
            int end = (i != len) ? i - 1 : i;
            double v;
            if (!fortran_real(line.substr(begin - 1, end - begin + 1), &v)) return false;
            ++num;
            a[set - 1][i1 - 1] = v;
            ++i1;
            if (num == 8) { i1 = 1; set = 1; }
          }
          begin = i;
        }
        prev = cl;
      }
    }
  }
  return found;
}

bool molar_mass(Deck& d, const std::string& name, double* w) {
  d.rewind();
  std::vector<std::string> v;
  while (!d.eof()) {
    if (!d.items(&v, 2) || v.size() < 2) return false;
    double x;
    if (!fortran_real(v[1], &x)) return false;
    if (same(v[0], name)) { *w = x; return true; }
  }
  return false;
}

// get_transport_properties (thermophysical_properties_class.f90:1379-1414):
// one header record, then READ(u,*) name, geometry, eps/k_B, sigma until the
// name matches; sigma is converted from Angstrom to nm.
bool transport_record(Deck& d, const std::string& name, double* eps, double* sigma) {
  d.rewind();
  std::string hdr;
  if (!d.item(&hdr)) return false;
  std::vector<std::string> v;
  while (true) {
    if (!d.items(&v, 4) || v.size() < 4) return false;
    char* end = nullptr;
    std::strtol(v[1].c_str(), &end, 10);
    if (v[1].empty() || *end != 0) return false;
    double e, sg;
    if (!fortran_real(v[2], &e) || !fortran_real(v[3], &sg)) return false;
    if (same(v[0], name)) {
      *eps = e;
      *sigma = sg * 0.1;
      return true;
    }
  }
}

}  // namespace

std::string load_transport(const std::string& transport_path, Mechanism* m) {
  Deck tr;
  if (!tr.open(transport_path)) return "cannot open transport file " + transport_path;
  const int n = m->n();
  m->well_depth.assign(n, 0.0);
  m->collision_diameter.assign(n, 0.0);
  for (int k = 0; k < n; ++k) {
    const std::string name = m->species[k].substr(0, 10);  // character(len=10) dummy
    if (!transport_record(tr, name, &m->well_depth[k], &m->collision_diameter[k]))
      return "transport data missing or unreadable for " + name;
  }
  // initialize_binary_diffusivity_constants (:1343-1377)
  m->binary_diffusivity.assign((size_t)n * n, 0.0);
  const std::vector<double>&W = m->molar_mass, &sg = m->collision_diameter;
  for (int i = 0; i < n - 1; ++i) {
    if (W[i] <= 0.0 || sg[i] <= 0.0) continue;
    for (int j = i + 1; j < n; ++j) {
      if (W[j] <= 0.0 || sg[j] <= 0.0) continue;
      double red = 0.5 * (sg[i] + sg[j]);
      red = red * red;
      const double inv_mu = (W[i] + W[j]) / (W[i] * W[j]);
      m->binary_diffusivity[(size_t)i * n + j] = 0.00001 * 0.595 * std::sqrt(inv_mu) / red;
      m->binary_diffusivity[(size_t)j * n + i] = m->binary_diffusivity[(size_t)i * n + j];
    }
  }
  return "";
}

std::string load_mechanism(const std::string& mech_path, const std::string& thermo_path,
                           const std::string& molar_path, double eff_default, EactUnits units,
                           Mechanism* out) {
  *out = Mechanism();
  Deck mech, thermo, molar;
  if (!mech.open(mech_path)) return "cannot open mechanism file " + mech_path;
  if (!read_species(mech, out)) return "species block not readable";
  std::string e = read_reactions(mech, eff_default, out);
  if (!e.empty()) return e;
  double coef = 1.0;
  switch (units) {
    case EactUnits::J_mol: coef = 1.0; break;
    case EactUnits::kJ_mol: coef = 1000.0; break;
    case EactUnits::cal_mol: coef = kRGasJ / kRGasCal; break;
    case EactUnits::kcal_mol: coef = kRGasJ / kRGasCal * 1000.0; break;
    default: return "unknown activation-energy units";
  }
  for (Reaction& rx : out->reactions) {
    if (rx.n_left == 2) rx.A = rx.A * 1.0e-06;
    if (rx.n_left == 3) rx.A = rx.A * 1.0e-12;
    if (rx.n_left + 1 == 2) rx.A_low = rx.A_low * 1.0e-06;
    if (rx.n_left + 1 == 3) rx.A_low = rx.A_low * 1.0e-12;
    rx.E = rx.E * coef;
    rx.E_low = rx.E_low * coef;
  }
  if (!thermo.open(thermo_path)) return "cannot open thermo file " + thermo_path;
  if (!molar.open(molar_path)) return "cannot open molar-mass file " + molar_path;
  const int n = out->n();
  out->a_coeffs.assign((size_t)n * 14, 0.0);
  out->molar_mass.assign(n, 0.0);
  for (int k = 0; k < n; ++k) {
    std::string name = out->species[k].substr(0, 10);  // character(len=10) dummy
    double a[2][7];
    if (!nasa7(thermo, name, a)) return "NASA-7 data missing or unreadable for " + name;
    for (int s = 0; s < 2; ++s)
      for (int i = 0; i < 7; ++i) out->a_coeffs[((size_t)k * 2 + s) * 7 + i] = a[s][i] * kRGasJ;
    if (!molar_mass(molar, name, &out->molar_mass[k])) return "molar mass missing for " + name;
  }
  return "";
}

static inline int coeff_set(double temp) { return temp >= 1000.0 ? 1 : 0; }

double specie_cp(const Mechanism& m, double T, int k) {
  double t = T < kTCeiling ? T : kTCeiling;
  const double* a = &m.a_coeffs[((size_t)k * 2 + coeff_set(t)) * 7];
  double cp = a[4];
  for (int i = 3; i >= 0; --i) cp = cp * t + a[i];
  return cp;
}

double specie_enthalpy(const Mechanism& m, double T, int k) {
  double t = T < kTCeiling ? T : kTCeiling;
  const double* a = &m.a_coeffs[((size_t)k * 2 + coeff_set(t)) * 7];
  double h = a[4] / 5.0;
  for (int i = 3; i >= 0; --i) h = h * t + a[i] / (double)(i + 1);
  h = h + a[5] / t;
  return h * t;
}

double specie_entropy(const Mechanism& m, double T, int k) {
  double t = T < kTCeiling ? T : kTCeiling;
  const double* a = &m.a_coeffs[((size_t)k * 2 + coeff_set(t)) * 7];
  double s = a[4] / 4.0;
  for (int i = 3; i >= 1; --i) s = s * t + a[i] / (double)i;
  return s * t + a[6] + a[0] * std::log(t);
}

}  // namespace nrg
