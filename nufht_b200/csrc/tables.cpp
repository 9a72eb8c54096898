// Planning tables of the NUFHT: Hankel coefficients a_k(nu), the asymptotic switch
// point z(nu, tol, K) and the Wimp expansion degree K_loc(nu, tol, K).
//
// Restates the defining formulas of the reference's table generator (src/bounds.c:63-297)
// and reads / writes its cache file format (src/fast_hankel_nufht.c:183-312), so that a
// cache produced by either library is accepted by the other.  Lookup order for the cache
// follows src/fast_hankel_nufht.c:95-179 ($NUFHT_TABLE_CACHE, ./data, ../data, the
// executable's directory), then this library's own data directory; when no cache is
// found the tables are generated (about a second on one core) and saved there.
#include "nufht_internal.h"

#include <dlfcn.h>
#include <limits.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

// The reference exports its three tables as globals (src/fast_hankel_nufht.c:36-45);
// they are exported here with the same names, types and shapes.
extern "C" {
double ASY_COEF_TABLE[NUFHT_NU_ROWS][NUFHT_MAX_COEF];
double ASY_Z_TABLE[NUFHT_MAX_I][NUFHT_MAX_J][NUFHT_MAX_K];
int WIMP_K_TABLE[NUFHT_MAX_I][NUFHT_MAX_J][NUFHT_MAX_K];
}

namespace hankel {
namespace {

constexpr int kNuMax = 200;     // integer orders 0..200
constexpr int kMaxAsyK = 10;    // asymptotic term counts 1..10 (src/bounds.c:46)
constexpr int kNTols = 12;      // tolerances 1e-4 .. 1e-15 (src/bounds.c:47-53)
const double kTols[kNTols] = {1e-4, 1e-5, 1e-6, 1e-7, 1e-8, 1e-9,
                              1e-10, 1e-11, 1e-12, 1e-13, 1e-14, 1e-15};

// a_k(nu) = prod_{j odd <= 2k-1} (4 nu^2 - j^2) / (k! 8^k)   (src/bounds.c:63-82)
double hankel_a(int k, double nu) {
  if (k == 0) return 1.0;
  double prod = 1.0;
  for (int j = 1; j <= 2 * k - 1; j += 2) prod *= 4.0 * nu * nu - (double)(j * j);
  double fact = 1.0;
  for (int j = 2; j <= k; ++j) fact *= (double)j;
  return prod / (fact * std::pow(8.0, (double)k));
}

// Size of the first omitted pair of Hankel terms with K terms kept (src/bounds.c:120-131).
double asy_bound(double nu, int K, double z) {
  double a1 = std::fabs(hankel_a(2 * K, nu)), a2 = std::fabs(hankel_a(2 * K + 1, nu));
  double z1 = std::pow(z, (double)(2 * K)), z2 = std::pow(z, (double)(2 * K + 1));
  return std::sqrt(2.0 / (M_PI * z)) * (a1 / z1 + a2 / z2);
}

// Newton iteration with a central-difference slope for asy_bound(z) = tol, from z = 1,
// relative step tolerance 1e-8, at most 1000 steps (src/bounds.c:141-175).
double asy_switch_point(double nu, int K, double tol) {
  double x = 1.0;
  for (int it = 0; it < 1000; ++it) {
    double f = asy_bound(nu, K, x) - tol;
    double h = 1e-5 * (std::fabs(x) > 1.0 ? std::fabs(x) : 1.0);
    double fp = asy_bound(nu, K, x + h) - tol;
    double fm = asy_bound(nu, K, x - h) - tol;
    double df = (fp - fm) / (2.0 * h);
    if (std::fabs(df) < 1e-16) break;
    double dx = -f / df;
    x += dx;
    if (x <= 0.0) x = std::fabs(x);
    if (std::fabs(dx / x) <= 1e-8) break;
  }
  return x;
}

double psi(double p) {  // src/bounds.c:223-228
  double r = std::sqrt(std::fmax(0.0, 1.0 - p * p));
  return std::log(p) + r - std::log(1.0 + r);
}

// Truncation bound of the Wimp expansion with K terms at argument z (src/bounds.c:230-250).
double wimp_bound(double nu, int K, double z) {
  double bK = psi(z / (2.0 * K + 2.0 + nu));
  double tkm = 2.0 * K - nu;
  if (tkm > 0.0 && z / tkm <= 1.0) {
    double cK = psi(z / (2.0 * K + 2.0 - nu));
    return 2.0 * std::exp(bK * (nu / 2.0 + K + 1.0) + cK * (-nu / 2.0 + K + 1.0)) /
           (1.0 - std::exp(bK + cK));
  }
  return 2.0 * std::exp(bK * (nu / 2.0 + K + 1.0)) / (1.0 - std::exp(bK));
}

void fill(Tables* T, int max_asy_K) {
  std::memset(T, 0, sizeof(*T));
  // Coefficient rows for nu = 0, 0.5, ..., 200, J = 0..2*10+1 (src/bounds.c:93-112).
  for (int i = 0; i <= 2 * kNuMax; ++i)
    for (int J = 0; J <= 2 * kMaxAsyK + 1; ++J) T->coef[i][J] = hankel_a(J, 0.5 * i);
  for (int nu = 0; nu <= kNuMax; ++nu)
    for (int j = 0; j < kNTols; ++j)
      for (int K = 1; K <= max_asy_K; ++K) {
        double z = asy_switch_point((double)nu, K, kTols[j]);
        T->z[nu][j][K - 1] = z;
        // Smallest Wimp degree whose bound is below tol (src/bounds.c:266-297).
        int wk = (int)std::ceil((z - (double)nu) / 2.0);
        if (wk < 1) wk = 1;
        for (int guard = 0; guard < 1000000 && !(wimp_bound((double)nu, wk, z) < kTols[j]);
             ++guard)
          ++wk;
        T->kw[nu][j][K - 1] = wk;
      }
}

bool file_is_dir(const std::string& p) {
  struct stat st;
  return stat(p.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

std::string library_dir() {
  Dl_info info;
  if (dladdr((void*)&library_dir, &info) && info.dli_fname) {
    std::string p(info.dli_fname);
    size_t s = p.rfind('/');
    if (s != std::string::npos) return p.substr(0, s);
  }
  return ".";
}

std::once_flag g_once;
Tables* g_tables = nullptr;
Tables* g_ext_tables = nullptr;
std::once_flag g_ext_once;
std::string g_source;

void publish_globals(const Tables* T) {
  std::memcpy(ASY_COEF_TABLE, T->coef, sizeof(T->coef));
  std::memcpy(ASY_Z_TABLE, T->z, sizeof(T->z));
  std::memcpy(WIMP_K_TABLE, T->kw, sizeof(T->kw));
}

void init_tables() {
  Tables* T = new Tables;
  std::string found;
  std::vector<std::string> cands;
  if (const char* env = std::getenv("NUFHT_TABLE_CACHE")) {
    cands.push_back(env);
  } else {
    char cwd[PATH_MAX];
    if (getcwd(cwd, sizeof cwd)) {
      std::string c(cwd);
      if (file_is_dir(c + "/data")) cands.push_back(c + "/data/nufht_tables.cache");
      size_t s = c.rfind('/');
      if (s != std::string::npos && file_is_dir(c.substr(0, s) + "/data"))
        cands.push_back(c.substr(0, s) + "/data/nufht_tables.cache");
    }
    char exe[PATH_MAX];
    ssize_t r = readlink("/proc/self/exe", exe, sizeof(exe) - 1);
    if (r > 0) {
      exe[r] = 0;
      std::string e(exe);
      size_t s = e.rfind('/');
      if (s != std::string::npos) cands.push_back(e.substr(0, s) + "/data/nufht_tables.cache");
    }
  }
  std::string own = library_dir() + "/data/nufht_tables.cache";
  cands.push_back(own);
  for (const auto& p : cands)
    if (tables_load(T, p.c_str()) == 0) { found = p; break; }
  if (found.empty()) {
    fill(T, kMaxAsyK);
    std::string save = std::getenv("NUFHT_TABLE_CACHE") ? std::getenv("NUFHT_TABLE_CACHE") : own;
    if (tables_save(T, save.c_str()) != 0)
      std::fprintf(stderr, "nufht_b200: could not save tables to %s\n", save.c_str());
    found = "generated";
  }
  g_source = found;
  publish_globals(T);
  g_tables = T;
}

}  // namespace

int tables_load(Tables* T, const char* path) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return -2;
  uint32_t h[6];
  if (std::fread(h, sizeof(uint32_t), 6, f) != 6) { std::fclose(f); return -3; }
  if (h[0] != 0x4E5546u || h[1] != 1u || h[2] != NUFHT_NU_ROWS || h[3] != NUFHT_MAX_I ||
      h[4] != NUFHT_MAX_J || h[5] != NUFHT_MAX_K) {
    std::fclose(f);
    return -4;
  }
  size_t n1 = sizeof(T->coef) / sizeof(double), n2 = sizeof(T->z) / sizeof(double),
         n3 = sizeof(T->kw) / sizeof(int);
  int rc = 0;
  if (std::fread(T->coef, sizeof(double), n1, f) != n1) rc = -5;
  else if (std::fread(T->z, sizeof(double), n2, f) != n2) rc = -6;
  else if (std::fread(T->kw, sizeof(int), n3, f) != n3) rc = -7;
  std::fclose(f);
  return rc;
}

int tables_save(const Tables* T, const char* path) {
  FILE* f = std::fopen(path, "wb");
  if (!f) return -2;
  uint32_t h[6] = {0x4E5546u, 1u, NUFHT_NU_ROWS, NUFHT_MAX_I, NUFHT_MAX_J, NUFHT_MAX_K};
  bool ok = std::fwrite(h, sizeof(uint32_t), 6, f) == 6 &&
            std::fwrite(T->coef, sizeof(T->coef), 1, f) == 1 &&
            std::fwrite(T->z, sizeof(T->z), 1, f) == 1 &&
            std::fwrite(T->kw, sizeof(T->kw), 1, f) == 1;
  std::fclose(f);
  return ok ? 0 : -3;
}

const Tables* tables() {
  std::call_once(g_once, init_tables);
  return g_tables;
}

// Same tables with the asymptotic switch point and Wimp degree also filled for eleven
// kept terms (index 10), which planning reads for K_asy = 10 (|nu| >= 35 at tol 1e-8).
const Tables* tables_extended() {
  std::call_once(g_ext_once, [] {
    const Tables* base = tables();
    Tables* T = new Tables;
    std::memcpy(T, base, sizeof(Tables));
    for (int nu = 0; nu <= kNuMax; ++nu)
      for (int j = 0; j < kNTols; ++j) {
        int K = kMaxAsyK + 1;
        double z = asy_switch_point((double)nu, K, kTols[j]);
        T->z[nu][j][K - 1] = z;
        int wk = (int)std::ceil((z - (double)nu) / 2.0);
        if (wk < 1) wk = 1;
        for (int guard = 0; guard < 1000000 && !(wimp_bound((double)nu, wk, z) < kTols[j]);
             ++guard)
          ++wk;
        T->kw[nu][j][K - 1] = wk;
      }
    g_ext_tables = T;
  });
  return g_ext_tables;
}

const char* tables_source() {
  tables();
  return g_source.c_str();
}

void tables_regenerate_into(Tables* T) { fill(T, kMaxAsyK); }

}  // namespace hankel

extern "C" void generate_tables(void) {
  // Regenerate from the formulas and publish into the exported globals.
  hankel::Tables* T = new hankel::Tables;
  hankel::tables_regenerate_into(T);
  std::memcpy(ASY_COEF_TABLE, T->coef, sizeof(T->coef));
  std::memcpy(ASY_Z_TABLE, T->z, sizeof(T->z));
  std::memcpy(WIMP_K_TABLE, T->kw, sizeof(T->kw));
  delete T;
}

// Write freshly generated tables to `path` in the cache format (used by the build step).
extern "C" int nufht_b200_write_tables(const char* path) {
  hankel::Tables* T = new hankel::Tables;
  hankel::tables_regenerate_into(T);
  int rc = hankel::tables_save(T, path);
  delete T;
  return rc;
}
