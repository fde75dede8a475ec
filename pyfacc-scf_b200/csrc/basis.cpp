// Basis construction from Basis-Set-Exchange "Gaussian94" text files.
//
// Shell order follows build_basis / read_shell / read_sp_shell of
// PyFAcc-SCF (src/fortran/basis.f90:9-190): element sections in file order,
// shell lines in section order, matching atoms in input order; an SP line
// yields the S shells of all matching atoms, then their P shells.
// Contraction coefficients are used as printed (no renormalisation of the
// contracted functions).  Sections are delimited by '****', so shell lines
// of absent elements are never mistaken for element labels (basis.f90:30-60
// would read an 'S' shell line as sulphur).  D lines (Sc and heavier), which
// basis.f90:76-82 has no branch for, become Cartesian d shells (xx, xy, xz,
// yy, yz, zz, each component normalised on its own, as the oracle reads
// them); other shell types are rejected with PYFACC_ERR_UNSUPPORTED_L
// instead of being misparsed.
#include <dlfcn.h>
#include <sys/stat.h>

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>

#include "engine.h"
#include "pool.h"

namespace pyfacc {

static const char* kSymbols[] = {
    "",   "H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al",
    "Si", "P",  "S",  "Cl", "Ar", "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co",
    "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr", "Rb", "Sr", "Y",  "Zr", "Nb",
    "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I",  "Xe"};
static const int kNumElements = 54;  // periodic_table of helper_functions.py:10-19

const char* element_symbol(int z) { return (z >= 1 && z <= kNumElements) ? kSymbols[z] : ""; }

int element_z(const std::string& sym) {
  for (int z = 1; z <= kNumElements; ++z)
    if (sym == kSymbols[z]) return z;
  return 0;
}

static bool file_exists(const std::string& p) {
  struct stat st;
  return stat(p.c_str(), &st) == 0 && S_ISREG(st.st_mode);
}

static std::string library_dir() {
  Dl_info info;
  if (dladdr(reinterpret_cast<void*>(&library_dir), &info) && info.dli_fname) {
    std::string p = info.dli_fname;
    size_t k = p.rfind('/');
    if (k != std::string::npos) return p.substr(0, k);
  }
  return ".";
}

// ./data/basis_set/<name>.txt first (main.f90:33), then the options'
// data_dir, then $PYFACC_DATA_DIR, then the data shipped beside the library.
std::string resolve_basis_file(const std::string& name, const char* data_dir) {
  std::vector<std::string> cands;
  if (data_dir && *data_dir) cands.push_back(std::string(data_dir) + "/basis_set/" + name + ".txt");
  cands.push_back("./data/basis_set/" + name + ".txt");
  if (const char* env = std::getenv("PYFACC_DATA_DIR")) cands.push_back(std::string(env) + "/basis_set/" + name + ".txt");
  cands.push_back(library_dir() + "/../data/basis_set/" + name + ".txt");
  for (const auto& c : cands)
    if (file_exists(c)) return c;
  throw Error(PYFACC_ERR_BASIS_NOT_FOUND, "basis set file for '" + name + "' not found");
}

static double parse_num(std::string tok) {
  for (auto& ch : tok)
    if (ch == 'D' || ch == 'd') ch = 'E';
  return std::strtod(tok.c_str(), nullptr);
}

static std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

static std::vector<std::string> read_lines(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw Error(PYFACC_ERR_BASIS_NOT_FOUND, "cannot open " + path);
  std::vector<std::string> lines;
  for (std::string ln; std::getline(in, ln);) lines.push_back(ln);
  return lines;
}

// Shells of the given atoms without their centres (every shell's c is 0).
static Basis basis_template(const std::string& basis_file, const std::vector<std::string>& species) {
  const auto text = basis_lines(basis_file, &read_lines);
  const std::vector<std::string>& lines = *text;
  Basis B;
  const int natoms = (int)species.size();
  std::vector<int> seen(natoms, 0);
  size_t i = 0;
  while (i < lines.size()) {
    const std::string ln = lines[i++];
    const std::string t = trim(ln);
    if (t.empty() || ln[0] == '!') continue;
    std::istringstream ss(t);
    std::string label;
    ss >> label;
    if (label == "****") continue;
    std::vector<int> atoms;
    for (int a = 0; a < natoms; ++a)
      if (species[a] == label) atoms.push_back(a);
    while (i < lines.size()) {
      const std::string sl = lines[i++];
      if (sl.find("****") != std::string::npos) break;
      if (atoms.empty() || trim(sl).empty()) continue;
      std::istringstream hs(sl);
      std::string kind;
      int nprim = 0;
      hs >> kind >> nprim;
      if (kind != "S" && kind != "P" && kind != "SP" && kind != "D")
        throw Error(PYFACC_ERR_UNSUPPORTED_L,
                    "shell type '" + kind + "' of " + label + " is not supported (S, P, SP and D only)");
      if (nprim <= 0 || i + nprim > lines.size()) throw Error(PYFACC_ERR_INVALID, "truncated basis section for " + label);
      std::vector<double> ex(nprim), cs(nprim), cp(nprim);
      for (int k = 0; k < nprim; ++k) {
        std::istringstream ps(lines[i++]);
        std::string t0, t1, t2;
        ps >> t0 >> t1 >> t2;
        ex[k] = parse_num(t0);
        cs[k] = parse_num(t1);
        cp[k] = (kind == "SP") ? parse_num(t2) : 0.0;
      }
      auto emit = [&](int l, const std::vector<double>& c) {
        for (int a : atoms) {
          Shell s;
          s.l = l;
          s.atom = a;
          s.ex = ex;
          s.co = c;
          B.shells.push_back(std::move(s));
          seen[a] = 1;
        }
      };
      if (kind == "S") emit(0, cs);
      else if (kind == "P") emit(1, cs);
      else if (kind == "D") emit(2, cs);  // Cartesian xx, xy, xz, yy, yz, zz; basis.f90 has no D branch
      else {
        emit(0, cs);
        emit(1, cp);
      }
    }
  }
  for (int a = 0; a < natoms; ++a)
    if (!seen[a]) throw Error(PYFACC_ERR_ELEMENT, "no basis functions for element '" + species[a] + "'");
  B.bf_off.assign(B.shells.size() + 1, 0);
  for (size_t s = 0; s < B.shells.size(); ++s) {
    const int l = B.shells[s].l;
    B.bf_off[s + 1] = B.bf_off[s] + (l + 1) * (l + 2) / 2;
  }
  B.nbf = B.bf_off.back();
  return B;
}

// The shell list depends on the basis file and the species sequence only,
// so it is parsed once per (file, species) and copied with the centres
// filled in: batches of many molecules of few compositions (water clusters
// of 4..16 monomers) parse the file a dozen times instead of once per
// molecule.  Failed parses are not kept, so their errors repeat.
Basis build_basis(const std::string& basis_file, const std::vector<std::string>& species,
                  const std::vector<double>& xyz) {
  static std::mutex mu;
  static std::map<std::string, std::shared_ptr<const Basis>> cache;
  std::string key = basis_file;
  key.push_back('\n');
  for (const auto& s : species) {
    key += s;
    key.push_back(' ');
  }
  std::shared_ptr<const Basis> t;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) t = it->second;
  }
  if (!t) {
    t = std::make_shared<const Basis>(basis_template(basis_file, species));
    std::lock_guard<std::mutex> lk(mu);
    if (cache.size() >= 256) cache.clear();
    cache[key] = t;
  }
  Basis B = *t;
  for (auto& s : B.shells)
    for (int x = 0; x < 3; ++x) s.c[x] = xyz[3 * s.atom + x];
  return B;
}

}  // namespace pyfacc
