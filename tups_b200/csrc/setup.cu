// Host-side set-up: prms parsing, index/symmetry/form-factor tables, device
// allocation.  Follows SRC/parquet_ini.f90:289-374, SRC/parquet_util.f90:14-478,
// SRC/parquet_formfactors.f90 and SRC/preprocessing.f90:100-133.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "tups_internal.h"

using tups::cplx;
using tups::NS;

namespace tups {

int set_error(tups_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

int exchange(tups_ctx* ctx, int what, double* dev, size_t n, int op) {
  if (ctx->ntasks <= 1) return TUPS_OK;
  if (!ctx->xfn) return set_error(ctx, TUPS_ERR_STATE, "sharded context without an exchange function");
  int rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "exchange");
  if (rc) return rc;
  if (ctx->xfn(ctx->xuser, what, dev, n, op) != 0)
    return set_error(ctx, TUPS_ERR_COMM, "exchange " + std::to_string(what) + " between ranks failed");
  return TUPS_OK;
}

int cuda_check(tups_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return TUPS_OK;
  return set_error(ctx, e == cudaErrorMemoryAllocation ? TUPS_ERR_OOM : TUPS_ERR_CUDA,
                   std::string(what) + ": " + cudaGetErrorString(e));
}

int after_launch(tups_ctx* ctx, const char* name) {
  ctx->launches++;
  return cuda_check(ctx, cudaGetLastError(), name);
}

}  // namespace tups

namespace {

// ---- prms parsing: one list-directed item per record ----------------------
std::string first_item(const std::string& line) {
  size_t i = 0;
  while (i < line.size() && std::isspace((unsigned char)line[i])) i++;
  if (i < line.size() && (line[i] == '"' || line[i] == '\'')) {
    char q = line[i];
    size_t j = line.find(q, i + 1);
    return line.substr(i + 1, j == std::string::npos ? std::string::npos : j - i - 1);
  }
  size_t j = i;
  while (j < line.size() && !std::isspace((unsigned char)line[j]) && line[j] != ',' && line[j] != '/') j++;
  return line.substr(i, j - i);
}

bool parse_real(const std::string& t, double* v) {
  std::string s = t;
  for (auto& c : s)
    if (c == 'd' || c == 'D') c = 'e';
  char* end = nullptr;
  *v = std::strtod(s.c_str(), &end);
  return end && end != s.c_str() && *end == '\0';
}

bool parse_int(const std::string& t, int* v) {
  char* end = nullptr;
  long x = std::strtol(t.c_str(), &end, 10);
  if (!end || end == t.c_str() || *end != '\0') return false;
  *v = (int)x;
  return true;
}

bool parse_logical(const std::string& t, int* v) {
  size_t i = 0;
  while (i < t.size() && t[i] == '.') i++;
  if (i >= t.size()) return false;
  char c = (char)std::toupper((unsigned char)t[i]);
  if (c == 'T') { *v = 1; return true; }
  if (c == 'F') { *v = 0; return true; }
  return false;
}

// ---- lattice helpers (1-based like the reference) ---------------------------
inline int wrap_neg(int i, int N) { return ((-(i - 1) + N) % N) + 1; }

// symmetry_operation (SRC/parquet_util.f90:896-978)
void sym_op(int s, int ix, int iy, int N, int* ox, int* oy) {
  switch (s) {
    case 1: *ox = ix; *oy = iy; break;
    case 2: *ox = ix; *oy = wrap_neg(iy, N); break;
    case 3: *ox = wrap_neg(ix, N); *oy = iy; break;
    case 4: *ox = wrap_neg(ix, N); *oy = wrap_neg(iy, N); break;
    case 5: *ox = iy; *oy = ix; break;
    case 6: *ox = iy; *oy = wrap_neg(ix, N); break;
    case 7: *ox = wrap_neg(iy, N); *oy = wrap_neg(ix, N); break;
    default: *ox = wrap_neg(iy, N); *oy = ix; break;
  }
}

// symmetry_operation_inv (SRC/parquet_util.f90:982-1136): 6 and 8 swapped
void sym_op_inv(int s, int ix, int iy, int N, int* ox, int* oy) {
  sym_op(s == 6 ? 8 : (s == 8 ? 6 : s), ix, iy, N, ox, oy);
}

// list_symmetries (SRC/parquet_util.f90:1140-1207)
void list_symmetries(int kx, int ky, int nxibz, int out[8]) {
  for (int i = 0; i < 8; i++) out[i] = 0;
  if ((kx == 1 && ky == 1) || (kx == nxibz && ky == nxibz)) {
    out[0] = 1;
  } else if (kx == nxibz && ky == 1) {
    out[0] = out[4] = 1;
  } else if (kx == nxibz && ky > 1 && ky < nxibz) {
    out[0] = out[1] = out[4] = out[7] = 1;
  } else if (kx > 1 && ky < nxibz) {
    if (ky == 1) {
      out[0] = out[2] = out[4] = out[5] = 1;
    } else if (ky == kx) {
      out[0] = out[1] = out[2] = out[3] = 1;
    } else {
      for (int i = 0; i < 8; i++) out[i] = 1;
    }
  }
}

// character table, SRC/parquet_formfactors.f90:572-588: chr(i, rep), 1-based
const int CHAR_TABLE[5][8] = {{1, 1, 1, 1, 1, 1, 1, 1},
                              {1, -1, -1, 1, -1, 1, -1, 1},
                              {1, 1, 1, 1, -1, -1, -1, -1},
                              {1, -1, -1, 1, 1, -1, 1, -1},
                              {2, 0, 0, -2, 0, 0, 0, 0}};
inline int chr(int i, int rep) { return CHAR_TABLE[rep - 1][i - 1]; }

// sym_op_L (SRC/parquet_util.f90:732-890), 1-based l
bool sym_op_L(int is, int l_in, const std::vector<int>& reps, int* l_sym, double* fac) {
  int rep = reps[l_in - 1];
  if (rep >= 1 && rep <= 4) {
    *l_sym = l_in;
    *fac = chr(is, rep);
    return true;
  }
  if (rep == 5) {
    if (l_in <= 5) {
      static const int f[8] = {1, 1, -1, -1, 1, 1, -1, -1};
      *l_sym = is <= 4 ? l_in : l_in + 1;
      *fac = f[is - 1];
    } else {
      static const int f[8] = {1, -1, 1, -1, 1, 1, -1, -1};
      static const int dl[8] = {0, 1, 1, 0, 0, 1, 0, 1};
      *l_sym = l_in + dl[is - 1];
      *fac = f[is - 1];
    }
    return true;
  }
  if (rep == 6) {
    if (l_in <= 5) {
      static const int f[8] = {1, -1, 1, -1, 1, -1, -1, 1};
      *l_sym = is <= 4 ? l_in : l_in - 1;
      *fac = f[is - 1];
    } else {
      static const int f[8] = {1, -1, 1, -1, -1, -1, 1, 1};
      static const int dl[8] = {0, -1, -1, 0, 0, -1, 0, -1};
      *l_sym = l_in + dl[is - 1];
      *fac = f[is - 1];
    }
    return true;
  }
  return false;
}

// create_list + sort (SRC/parquet_formfactors.f90:594-646)
std::vector<int> create_list(int Nx) {
  std::vector<int> t;
  for (int i = 1; i <= Nx / 2 + 1; i++)
    for (int j = 1; j <= i; j++) {
      t.push_back(i - 1);
      t.push_back(j - 1);
      t.push_back((i - 1) * (i - 1) + (j - 1) * (j - 1));
    }
  int many = (int)t.size() / 3;
  for (int i = 1; i <= many; i++)
    for (int j = i; j >= 2; j--)
      if (t[3 * (j - 1) + 2] < t[3 * (j - 2) + 2])
        for (int c = 0; c < 3; c++) std::swap(t[3 * (j - 1) + c], t[3 * (j - 2) + c]);
  return t;
}

// Init_Formfactor_variables (SRC/parquet_formfactors.f90:451-537)
int init_nl(tups_ctx* ctx, const std::vector<int>& tl, std::vector<int>& pick) {
  const int Nx = ctx->p.Nx, Ny = Nx, npos = Nx * Ny;
  pick.assign(npos, 0);
  int Nl = 0;
  if (ctx->p.readinpick) {
    std::ifstream in(ctx->p.pick_file);
    if (!in) return tups::set_error(ctx, TUPS_ERR_IO, std::string("cannot open picklist ") + ctx->p.pick_file);
    std::string line;
    int i = 0;
    while (i < npos && std::getline(in, line)) {
      std::string tok = first_item(line);
      if (tok.empty()) continue;
      int v;
      if (!parse_logical(tok, &v)) return tups::set_error(ctx, TUPS_ERR_IO, "bad picklist entry " + tok);
      pick[i++] = v;
      Nl += v;
    }
    if (i < npos) return tups::set_error(ctx, TUPS_ERR_IO, "picklist shorter than Nx*Ny");
    return Nl;
  }
  int many = (int)tl.size() / 3;
  if (ctx->p.neighbours < 1 || ctx->p.neighbours > many)
    return tups::set_error(ctx, TUPS_ERR_BADDIM, "neighbours out of range");
  for (int i = 0; i < ctx->p.neighbours; i++) {
    int x = tl[3 * i], y = tl[3 * i + 1];
    if (x == 0 && y == 0) Nl += 1;
    else if (std::fabs(x - Nx / 2.0) < 0.01 && std::fabs(y - Ny / 2.0) < 0.01) Nl += 1;
    else if (std::fabs(x - Nx / 2.0) < 0.01 && y == 0) Nl += 2;
    else if (std::fabs(x - Nx / 2.0) < 0.01) Nl += 4;
    else if (x == y || y == 0) Nl += 4;
    else Nl += 8;
  }
  for (int i = 0; i < npos; i++) pick[i] = i < Nl ? 1 : 0;
  return Nl;
}

// initialize_bonds (SRC/parquet_formfactors.f90:95-360)
bool initialize_bonds(int Nx, int Nl, const std::vector<int>& tl, const std::vector<int>& pick,
                      std::vector<int>& bonds, std::vector<int>& signs, std::vector<int>& reps) {
  const int Ny = Nx;
  bonds.assign(3 * Nl, 0);
  signs.assign(Nl, 1);
  reps.assign(Nl, 0);
  const int c41[4] = {1, 4, 5, 5}, c42[4] = {1, 3, 5, 5}, c8[8] = {1, 2, 3, 4, 5, 5, 5, 5};
  int b = 1, lg = 1, lat = 1;
  const int many = (int)tl.size() / 3, npick = (int)pick.size();
  auto picked = [&](int pos) { return pos >= 1 && pos <= npick && pick[pos - 1]; };
  // returns true when all Nl bonds are placed
  auto put = [&](int bx, int by, int ch, int rep, int sgn) {
    bonds[3 * (b - 1)] = bx;
    bonds[3 * (b - 1) + 1] = by;
    bonds[3 * (b - 1) + 2] = ch;
    reps[b - 1] = rep;
    if (sgn) signs[b - 1] = sgn;
    b++;
    return b > Nl;
  };
  while (true) {
    if (lat > many) return false;
    int x = tl[3 * (lat - 1)], y = tl[3 * (lat - 1) + 1];
    if (x == 0 && y == 0) {
      if (picked(lg) && put(x, y, 1, 1, 0)) break;
      lg++; lat++;
      continue;
    } else if (std::fabs(x - Nx / 2.0) < 0.01 && std::fabs(y - Ny / 2.0) < 0.01) {
      if (picked(lg) && put(x, y, 1, 1, 0)) break;
      lg++; lat++;
      continue;
    } else if (std::fabs(x - Nx / 2.0) < 0.01 && y == 0) {
      if (picked(lg) && put(x, y, 1, 1, 0)) break;
      lg++;
      if (picked(lg) && put(x, y, 3, 3, 0)) break;
      lg++; lat++;
      continue;
    } else if (x == y) {
      bool done = false;
      for (int i = 1; i <= 3 && !done; i++) {
        if (picked(lg) && put(x, y, c41[i - 1], c41[i - 1], i == 3 ? -1 : 0)) { done = true; break; }
        lg++;
      }
      if (done) break;
      if (picked(lg) && put(-y, x, c41[3], 6, -1)) break;
      lg++; lat++;
      continue;
    } else if (y == 0 || std::fabs(x - Nx / 2.0) < 0.01) {
      bool done = false;
      for (int i = 1; i <= 3 && !done; i++) {
        if (picked(lg) && put(x, y, c42[i - 1], c42[i - 1], i == 3 ? -1 : 0)) { done = true; break; }
        lg++;
      }
      if (done) break;
      // the DO variable is 4 after the loop completes: chars_42(4)
      if (picked(lg) && put(-y, x, c42[3], 6, -1)) break;
      lg++; lat++;
      continue;
    } else {
      bool done = false;
      for (int i = 1; i <= 5 && !done; i++) {
        if (picked(lg) && put(x, y, c8[i - 1], c8[i - 1], i == 5 ? -1 : 0)) { done = true; break; }
        lg++;
      }
      if (done) break;
      if (picked(lg) && put(x, -y, c8[5], 6, -1)) break;
      lg++;
      if (picked(lg) && put(y, x, c8[6], 5, -1)) break;
      lg++;
      if (picked(lg) && put(-y, x, c8[7], 6, -1)) break;
      lg++; lat++;
      continue;
    }
  }
  return true;
}

// my_symmetry_operation (SRC/parquet_formfactors.f90:367-446), no wrap
void my_sym(int s, int x, int y, int* ox, int* oy) {
  switch (s) {
    case 1: *ox = x; *oy = y; break;
    case 2: *ox = x; *oy = -y; break;
    case 3: *ox = -x; *oy = y; break;
    case 4: *ox = -x; *oy = -y; break;
    case 5: *ox = y; *oy = x; break;
    case 6: *ox = y; *oy = -x; break;
    case 7: *ox = -y; *oy = -x; break;
    default: *ox = -y; *oy = x; break;
  }
}

// FF_array (SRC/parquet_formfactors.f90:11-90): FF(kx,ky,l) column-major
void ff_array(int Nx, int Nl, const std::vector<int>& bonds, std::vector<double>& FF) {
  const int Ny = Nx;
  std::vector<double> re((size_t)Nx * Ny * Nl, 0.0), im((size_t)Nx * Ny * Nl, 0.0);
  for (int l = 0; l < Nl; l++) {
    int x0 = bonds[3 * l], y0 = bonds[3 * l + 1], ch = bonds[3 * l + 2];
    int bx[8], by[8], bw[8];
    for (int i = 1; i <= 8; i++) {
      my_sym(i, x0, y0, &bx[i - 1], &by[i - 1]);
      bw[i - 1] = chr(i, ch);
    }
    for (int kx = 1; kx <= Nx; kx++)
      for (int ky = 1; ky <= Ny; ky++) {
        double ar = 0.0, ai = 0.0;
        for (int i = 0; i < 8; i++) {
          double px = 2.0 / Nx * M_PI * (kx - 1);
          double py = 2.0 / Ny * M_PI * (ky - 1);
          double ang = bx[i] * px + by[i] * py;
          ar = ar + bw[i] * std::cos(ang);
          ai = ai + bw[i] * std::sin(ang);
        }
        size_t idx = (size_t)(kx - 1) + (size_t)Nx * ((ky - 1) + (size_t)Ny * l);
        re[idx] = ar;
        im[idx] = ai;
      }
  }
  FF.assign((size_t)Nx * Ny * Nl, 0.0);
  for (int l = 0; l < Nl; l++) {
    double norm = 0.0;
    for (int kx = 0; kx < Nx; kx++)
      for (int ky = 0; ky < Ny; ky++) {
        size_t idx = kx + (size_t)Nx * (ky + (size_t)Ny * l);
        double a = std::hypot(re[idx], im[idx]);
        norm += a * a;
      }
    double inv = 1.0 / std::sqrt(norm);
    for (int kx = 0; kx < Nx; kx++)
      for (int ky = 0; ky < Ny; ky++) {
        size_t idx = kx + (size_t)Nx * (ky + (size_t)Ny * l);
        FF[idx] = inv * re[idx] + inv * im[idx];
      }
  }
}

template <typename T>
int dalloc(tups_ctx* ctx, T** ptr, size_t count) {
  *ptr = nullptr;
  if (count == 0) count = 1;
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, count * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return tups::set_error(ctx, TUPS_ERR_OOM,
                           "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed");
  }
  ctx->allocations.push_back(p);
  *ptr = (T*)p;
  return TUPS_OK;
}

template <typename T>
int upload(tups_ctx* ctx, T** ptr, const std::vector<T>& v) {
  int rc = dalloc(ctx, ptr, v.size());
  if (rc) return rc;
  return tups::cuda_check(ctx, cudaMemcpy(*ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice),
                          "upload");
}

}  // namespace

#define TRY(x)                      \
  do {                              \
    int _rc = (x);                  \
    if (_rc != TUPS_OK) return _rc; \
  } while (0)

// Optional extensions beside the reference's prms (no counterpart in the
// reference, whose 21 records stay as they are): `<prms>.gpu`, one
// `key = value` (or `key value`) per line, `!` or `#` starts a comment.
// Keys: tprime (the t' hopping), conv_abs (sup-norm convergence threshold on
// dSigma).  An absent file leaves both 0; an unknown key or a bad value is an
// error, so a misspelt key is not silently ignored.
static int read_prms_extras(const std::string& path, tups_params* p) {
  std::ifstream in(path);
  if (!in) return TUPS_OK;
  std::string line;
  while (std::getline(in, line)) {
    const size_t c = line.find_first_of("!#");
    if (c != std::string::npos) line.resize(c);
    for (auto& ch : line)
      if (ch == '=') ch = ' ';
    std::istringstream ls(line);
    std::string key, val, extra;
    if (!(ls >> key)) continue;
    if (!(ls >> val) || (ls >> extra)) return TUPS_ERR_IO;
    for (auto& ch : key) ch = (char)std::tolower((unsigned char)ch);
    double v;
    if (!parse_real(val, &v)) return TUPS_ERR_IO;
    if (key == "tprime") p->tprime = v;
    else if (key == "conv_abs") p->conv_abs = v;
    else return TUPS_ERR_IO;
  }
  return TUPS_OK;
}

extern "C" int tups_read_prms(const char* path, tups_params* out) {
  if (!path || !out) return TUPS_ERR_BADARG;
  std::ifstream in(path);
  if (!in) return TUPS_ERR_IO;
  std::vector<std::string> items;
  std::string line;
  while (items.size() < 21 && std::getline(in, line)) {
    std::string t = first_item(line);
    if (t.empty()) continue;
    items.push_back(t);
  }
  if (items.size() < 21) return TUPS_ERR_IO;
  tups_params p;
  std::memset(&p, 0, sizeof(p));
  bool ok = parse_real(items[0], &p.beta) && parse_real(items[1], &p.U) &&
            parse_real(items[2], &p.nParticle) && parse_int(items[3], &p.Nx) &&
            parse_int(items[4], &p.Nf) && parse_int(items[5], &p.neighbours) &&
            parse_logical(items[6], &p.readinpick) && parse_int(items[8], &p.Ngrain) &&
            parse_int(items[9], &p.f_range) && parse_real(items[10], &p.f_damping) &&
            parse_int(items[11], &p.ite_max) && parse_logical(items[12], &p.DGA) &&
            parse_logical(items[14], &p.use_sig_dmft) && parse_logical(items[16], &p.use_U2) &&
            parse_logical(items[17], &p.save_F) && parse_logical(items[18], &p.oneshot) &&
            parse_logical(items[19], &p.old) && parse_logical(items[20], &p.SDE_old);
  if (!ok) return TUPS_ERR_IO;
  std::snprintf(p.pick_file, sizeof(p.pick_file), "%s", items[7].c_str());
  std::snprintf(p.fname_L, sizeof(p.fname_L), "%s", items[13].c_str());
  std::snprintf(p.fname_sig_dmft, sizeof(p.fname_sig_dmft), "%s", items[15].c_str());
  const int rc = read_prms_extras(std::string(path) + ".gpu", &p);
  if (rc) return rc;
  *out = p;
  return TUPS_OK;
}

static int build_tables(tups_ctx* ctx) {
  const tups_params& p = ctx->p;
  tups_dims& d = ctx->d;
  if (p.Nx < 2 || p.Nx % 2) return tups::set_error(ctx, TUPS_ERR_BADDIM, "Nx must be even and >= 2");
  if (p.Nf < 6 || p.Nf % 2) return tups::set_error(ctx, TUPS_ERR_BADDIM, "Nf must be even and >= 6");
  if (p.Ngrain < 1) return tups::set_error(ctx, TUPS_ERR_BADDIM, "Ngrain must be >= 1");
  if (p.f_range < 0) return tups::set_error(ctx, TUPS_ERR_BADDIM, "f_range must be >= 0");
  if (p.old || p.SDE_old) return tups::set_error(ctx, TUPS_ERR_BADARG, "old PAE/SDE paths are not supported");
  d.Nx = d.Ny = p.Nx;
  d.Nf = p.Nf;
  d.Ngrain = p.Ngrain;
  d.Nx_IBZ = (p.Nx + 2) / 2;
  d.NIBZ = (d.Nx_IBZ * (d.Nx_IBZ + 1)) / 2;
  d.Nred = d.NIBZ * p.Nf / 2;
  d.Nc = p.Nx * p.Nx;
  d.Nt = d.Nc * p.Nf;
  d.Nb = d.Nred;
  d.wperTask = (p.Nf - 1) / 2 + 1;
  d.nbox = (2 * p.f_range + 1) * p.Nf;
  std::vector<int> tl = create_list(p.Nx);
  int Nl = init_nl(ctx, tl, ctx->pick);
  if (Nl < 0) return Nl;
  if (Nl < 1) return tups::set_error(ctx, TUPS_ERR_BADDIM, "no form factors selected");
  d.Nl = Nl;
  d.Nz = Nl * p.Nf;
  if (!initialize_bonds(p.Nx, Nl, tl, ctx->pick, ctx->bonds0, ctx->signs, ctx->reps))
    return tups::set_error(ctx, TUPS_ERR_BADDIM, "form-factor bond list exhausted");
  ff_array(p.Nx, Nl, ctx->bonds0, ctx->FF);
  d.NR = Nl == 1 ? 1 : (Nl == 5 ? 4 : (Nl == 9 ? 6 : 1));
  if (d.NR > d.NIBZ) return tups::set_error(ctx, TUPS_ERR_BADDIM, "NR exceeds NIBZ");
  const int Nx = d.Nx, Ny = d.Ny, Nf = d.Nf, Ng = d.Ngrain;
  // FF_inv (SRC/parquet_formfactors.f90:545-569), layout (8, Nx, Ny, Nl)
  ctx->FF_inv.assign((size_t)NS * Nx * Ny * Nl, 0.0);
  for (int l = 0; l < Nl; l++)
    for (int ky = 1; ky <= Ny; ky++)
      for (int kx = 1; kx <= Nx; kx++)
        for (int s = 1; s <= NS; s++) {
          int sx, sy;
          sym_op_inv(s, kx, ky, Nx, &sx, &sy);
          ctx->FF_inv[(s - 1) + NS * ((kx - 1) + (size_t)Nx * ((ky - 1) + (size_t)Ny * l))] =
              ctx->FF[(sx - 1) + (size_t)Nx * ((sy - 1) + (size_t)Ny * l)];
        }
  // l-space symmetry tables
  ctx->lsym.assign(NS * Nl, 0);
  ctx->lfac.assign(NS * Nl, 0.0);
  for (int s = 1; s <= NS; s++)
    for (int l = 1; l <= Nl; l++) {
      int ls;
      double f;
      if (!sym_op_L(s, l, ctx->reps, &ls, &f) || ls < 1 || ls > Nl)
        return tups::set_error(ctx, TUPS_ERR_BADDIM, "form-factor set not closed under the point group");
      ctx->lsym[(s - 1) + NS * (l - 1)] = ls - 1;
      ctx->lfac[(s - 1) + NS * (l - 1)] = f;
    }
  // index_bosonic_IBZ (SRC/parquet_util.f90:110-117)
  ctx->ibz.assign(3 * (size_t)d.Nred, 0);
  for (int kx = 1; kx <= d.Nx_IBZ; kx++)
    for (int ky = 1; ky <= kx; ky++)
      for (int w = 1; w <= Nf / 2; w++) {
        int idx = (((kx - 1) * kx) / 2 + ky - 1) * (Nf / 2) + w;
        ctx->ibz[3 * (idx - 1)] = kx;
        ctx->ibz[3 * (idx - 1) + 1] = ky;
        ctx->ibz[3 * (idx - 1) + 2] = w;
      }
  ctx->symlist.assign(NS * (size_t)d.NIBZ, 0);
  ctx->symq.assign(2 * NS * (size_t)d.NIBZ, 0);
  for (int iq = 0; iq < d.NIBZ; iq++) {
    int qx = ctx->ibz[3 * iq * (Nf / 2)], qy = ctx->ibz[3 * iq * (Nf / 2) + 1];
    list_symmetries(qx, qy, d.Nx_IBZ, &ctx->symlist[NS * iq]);
    for (int s = 1; s <= NS; s++) {
      int sx, sy;
      sym_op(s, qx, qy, Nx, &sx, &sy);
      ctx->symq[2 * (NS * iq + s - 1)] = sx;
      ctx->symq[2 * (NS * iq + s - 1) + 1] = sy;
    }
  }
  // dispersion (SRC/parquet_util.f90:128-164) plus the t' extension
  ctx->Ek.assign((size_t)Nx * Ny, 0.0);
  const double dkx = 2.0 * M_PI / Nx, dky = 2.0 * M_PI / Ny;
  for (int kx = 1; kx <= Nx; kx++) {
    double px = dkx * (kx - 1);
    for (int ky = 1; ky <= Ny; ky++) {
      double py = dky * (ky - 1);
      double e = 0.0;
      if (Nx > 1) e = e - 2.0 * std::cos(px);
      if (Ny > 1) e = e - 2.0 * std::cos(py);
      if (p.tprime != 0.0) e = e - 4.0 * p.tprime * std::cos(px) * std::cos(py);
      ctx->Ek[(kx - 1) + (size_t)Nx * (ky - 1)] = e;
    }
  }
  ctx->Ekg.assign((size_t)Ng * Ng * Nx * Ny, 0.0);
  for (int iy = 1; iy <= Ny; iy++)
    for (int ix = 1; ix <= Nx; ix++)
      for (int iy2 = 1; iy2 <= Ng; iy2++)
        for (int ix2 = 1; ix2 <= Ng; ix2++) {
          double px = dkx * (ix - 1) + (ix2 - (Ng + 1) / 2) * dkx / (double)Ng;
          double py = dky * (iy - 1) + (iy2 - (Ng + 1) / 2) * dky / (double)Ng;
          double e = 0.0 - 2.0 * std::cos(px) - 2.0 * std::cos(py);
          if (p.tprime != 0.0) e = e - 4.0 * p.tprime * std::cos(px) * std::cos(py);
          ctx->Ekg[(ix2 - 1) + (size_t)Ng * ((iy2 - 1) + (size_t)Ng * ((ix - 1) + (size_t)Nx * (iy - 1)))] = e;
        }
  if (d.Nc == 1) {
    std::fill(ctx->Ek.begin(), ctx->Ek.end(), 0.0);
    std::fill(ctx->Ekg.begin(), ctx->Ekg.end(), 0.0);
  }
  ctx->aux = std::fabs(1.0 / (ctx->FF[0] * ctx->FF[0]));
  return TUPS_OK;
}

// Fortran character variables are blank-padded: TRIM drops trailing blanks
static std::string trim_name(const char* c) {
  std::string t(c);
  while (!t.empty() && (t.back() == ' ' || t.back() == '\t')) t.pop_back();
  return t;
}

// DGA Lambda file (SRC/parquet_util.f90:321-343): Nf * Nf * Nf/2 records in
// the order k1 (slowest), k2, q (fastest), each read list-directed as
// "i i i re1 im1 re2 im2": a record may span lines, items left on its last
// line are skipped, commas separate like blanks.  The first complex number
// goes to A(k1, k2, q) (Lambda_d or Lambda_s), the second to B (Lambda_m or
// Lambda_t), both stored (Nf, Nf, Nf/2) column-major.
static int read_lambda_file(tups_ctx* ctx, const std::string& path, int Nf, std::vector<cplx>& A,
                            std::vector<cplx>& B) {
  std::ifstream in(path);
  if (!in) return tups::set_error(ctx, TUPS_ERR_IO, "cannot open " + path);
  const size_t nL = (size_t)Nf * Nf * (Nf / 2);
  A.assign(nL, make_double2(0.0, 0.0));
  B.assign(nL, make_double2(0.0, 0.0));
  std::string line;
  for (int k1 = 0; k1 < Nf; k1++)
    for (int k2 = 0; k2 < Nf; k2++)
      for (int q = 0; q < Nf / 2; q++) {
        std::vector<std::string> tok;
        while (tok.size() < 7 && std::getline(in, line)) {
          for (auto& c : line)
            if (c == ',') c = ' ';
          std::istringstream ls(line);
          std::string x;
          while (ls >> x) tok.push_back(x);
        }
        if (tok.size() < 7) return tups::set_error(ctx, TUPS_ERR_IO, path + ": file too short");
        int itemp;
        double v[4];
        bool ok = parse_int(tok[0], &itemp) && parse_int(tok[1], &itemp) && parse_int(tok[2], &itemp);
        for (int a = 0; a < 4; a++) ok = ok && parse_real(tok[3 + a], &v[a]);
        if (!ok) return tups::set_error(ctx, TUPS_ERR_IO, path + ": bad record");
        const size_t idx = (size_t)k1 + (size_t)Nf * (k2 + (size_t)Nf * q);
        A[idx] = make_double2(v[0], v[1]);
        B[idx] = make_double2(v[2], v[3]);
      }
  return TUPS_OK;
}

static int upload_tables(tups_ctx* ctx) {
  const tups_dims& d = ctx->d;
  auto& t = ctx->t;
  const int Nf = d.Nf, Nx = d.Nx, Ny = d.Ny, Ng = d.Ngrain;
  TRY(upload(ctx, &t.FF, ctx->FF));
  TRY(upload(ctx, &t.FF_inv, ctx->FF_inv));
  TRY(upload(ctx, &t.Ek, ctx->Ek));
  TRY(upload(ctx, &t.Ekg, ctx->Ekg));
  TRY(upload(ctx, &t.signs, ctx->signs));
  TRY(upload(ctx, &t.lsym, ctx->lsym));
  TRY(upload(ctx, &t.lfac, ctx->lfac));
  TRY(upload(ctx, &t.ibz, ctx->ibz));
  TRY(upload(ctx, &t.symlist, ctx->symlist));
  TRY(upload(ctx, &t.symq, ctx->symq));
  // Lambda (SRC/parquet_util.f90:311-346): constant per channel in the PA,
  // frequency-dependent tables from the two input files with DGA
  const double U = ctx->p.U;
  const double lam[4] = {U, -U, 2.0 * U, 0.0};
  size_t nL = (size_t)Nf * Nf * (Nf / 2);
  std::vector<cplx> Lr[4];
  if (ctx->p.DGA) {
    const std::string base = trim_name(ctx->p.fname_L);
    TRY(read_lambda_file(ctx, base + "_ph.init", Nf, Lr[0], Lr[1]));
    TRY(read_lambda_file(ctx, base + "_pp.init", Nf, Lr[2], Lr[3]));
  } else {
    for (int r = 0; r < 4; r++) Lr[r].assign(nL, make_double2(lam[r], 0.0));
  }
  for (int r = 0; r < 4; r++) TRY(upload(ctx, &t.L[r], Lr[r]));
  // twiddles: e^{i*(-pi/beta*(2(nu-Nf/2)-1))*tau} (SRC/parquet_chi.f90:161)
  {
    std::vector<cplx> tw((size_t)Nf * Nf);
    const double beta = ctx->p.beta;
    for (int it = 1; it <= Nf; it++) {
      double tau = beta / (Nf - 1) * (it - 1);
      for (int nu = 1; nu <= Nf; nu++) {
        double ph = -M_PI / beta * (2.0 * (nu - Nf / 2) - 1.0);
        double a = ph * tau;
        tw[(it - 1) + (size_t)Nf * (nu - 1)] = make_double2(std::cos(a), std::sin(a));
      }
    }
    TRY(upload(ctx, &t.tw_tau, tw));
  }
  for (int dim = 0; dim < 2; dim++) {
    int n = (dim == 0 ? Nx : Ny) * Ng;
    std::vector<cplx> tw(n);
    for (int m = 0; m < n; m++) {
      double a = -2.0 * M_PI * m / n;
      tw[m] = make_double2(std::cos(a), std::sin(a));
    }
    TRY(upload(ctx, dim == 0 ? &t.tw_x : &t.tw_y, tw));
  }
  return TUPS_OK;
}

static int alloc_state(tups_ctx* ctx) {
  const tups_dims& d = ctx->d;
  auto& s = ctx->s;
  const size_t Nt = d.Nt, Nz = d.Nz, Nb = d.Nb;
  const size_t ng2 = (size_t)d.Nx * d.Ngrain * d.Ny * d.Ngrain;
  TRY(dalloc(ctx, &s.Sigma, Nt));
  TRY(dalloc(ctx, &s.SigmaOld, Nt));
  TRY(dalloc(ctx, &s.SigmaH, (size_t)d.Nc));
  TRY(dalloc(ctx, &s.Gkw, Nt));
  TRY(dalloc(ctx, &s.Grt, ng2 * d.Nf));
  TRY(dalloc(ctx, &s.Grt_work, ng2 * d.Nf));
  for (int r = 0; r < 4; r++) {
    TRY(dalloc(ctx, &s.F[r], Nz * Nz * Nb));
    TRY(dalloc(ctx, &s.G[r], Nz * Nz * Nb));
    TRY(dalloc(ctx, &s.PhiR[r], Nz * Nz * (size_t)(d.Nf / 2) * d.NR));
    TRY(dalloc(ctx, &s.M[r], (size_t)d.Nl * d.Nl * d.Nl * d.Nl * d.NIBZ * d.NR));
  }
  TRY(dalloc(ctx, &s.chi_ph, (size_t)d.Nl * d.Nl * d.Nf * Nb));
  TRY(dalloc(ctx, &s.chi_pp, (size_t)d.Nl * d.Nl * d.Nf * Nb));
  // BSE scratch: Gamma*chi and chi*Gamma for a chunk of (q, channel) instances,
  // bounded to 4 GiB total
  size_t per = 2 * Nz * Nz * sizeof(cplx);
  size_t cap = ((size_t)4 << 30) / per;
  size_t want = 4 * Nb;
  s.bse_chunk = std::max<size_t>(4, std::min(want, cap)) / 4 * 4;
  TRY(dalloc(ctx, &s.bse_A, Nz * Nz * s.bse_chunk));
  TRY(dalloc(ctx, &s.bse_B, Nz * Nz * s.bse_chunk));
  TRY(dalloc(ctx, &ctx->t.expSqR, (size_t)d.NIBZ * d.NR * NS));
  TRY(dalloc(ctx, &ctx->t.expqSR, (size_t)d.Nc * d.NR * NS));
  TRY(dalloc(ctx, &s.chi_aux_ph, (size_t)d.Nl * d.nbox * Nb));
  TRY(dalloc(ctx, &s.chi_aux_pp, (size_t)d.Nl * d.nbox * Nb));
  TRY(dalloc(ctx, &s.LChi, Nz * Nb));
  TRY(dalloc(ctx, &s.PhChi, Nz * Nb));
  TRY(dalloc(ctx, &s.PPChi, Nz * Nb));
  TRY(dalloc(ctx, &s.SigmaV, (size_t)d.NIBZ * d.Nf));
  TRY(dalloc(ctx, &s.order2, Nt));
  TRY(dalloc(ctx, &s.GGG, ng2 * d.Nf));
  TRY(dalloc(ctx, &s.scal, (size_t)tups::S_COUNT));
  TRY(dalloc(ctx, &s.red, (size_t)1 << 16));
  return TUPS_OK;
}

// vertex initialisation (SRC/preprocessing.f90:100-116): F = G = Lambda(:, :, w)*Nc
// on the (l=1, l=1) nu-block of every bosonic slot; Sigma = 0 or the DMFT input
static int init_state(tups_ctx* ctx) {
  const tups_dims& d = ctx->d;
  auto& s = ctx->s;
  const size_t Nz = d.Nz, Nb = d.Nb;
  for (int r = 0; r < 4; r++) {
    const size_t bytes = Nz * Nz * Nb * sizeof(cplx);
    TRY(tups::cuda_check(ctx, cudaMemsetAsync(s.F[r], 0, bytes, ctx->stream), "init F"));
    TRY(tups::cuda_check(ctx, cudaMemsetAsync(s.G[r], 0, bytes, ctx->stream), "init G"));
    TRY(tups::launch_fill_lambda_block(ctx, s.F[r], s.G[r], ctx->t.L[r], ctx->aux));
  }
  TRY(tups::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "init vertices"));
  std::vector<cplx> sig((size_t)d.Nt, make_double2(0.0, 0.0));
  if (ctx->p.use_sig_dmft) {
    // SRC/parquet_util.f90:212-230: Sigma(k, nu) = i * (third column)
    std::ifstream in(ctx->p.fname_sig_dmft);
    if (!in) return tups::set_error(ctx, TUPS_ERR_IO, std::string("cannot open ") + ctx->p.fname_sig_dmft);
    std::vector<double> im;
    std::string line;
    while ((int)im.size() < d.Nf && std::getline(in, line)) {
      std::istringstream ls(line);
      std::string a, b, c;
      if (!(ls >> a >> b >> c)) continue;
      double x;
      if (!parse_real(c, &x)) return tups::set_error(ctx, TUPS_ERR_IO, "bad DMFT self-energy line");
      im.push_back(x);
    }
    if ((int)im.size() < d.Nf) return tups::set_error(ctx, TUPS_ERR_IO, "DMFT self-energy file too short");
    for (int k = 0; k < d.Nc; k++)
      for (int nu = 0; nu < d.Nf; nu++) sig[(size_t)k * d.Nf + nu] = make_double2(0.0, im[nu]);
  }
  TRY(tups::cuda_check(ctx, cudaMemcpy(s.Sigma, sig.data(), sig.size() * sizeof(cplx), cudaMemcpyHostToDevice),
                       "init Sigma"));
  TRY(tups::cuda_check(ctx, cudaMemcpy(s.SigmaOld, sig.data(), sig.size() * sizeof(cplx), cudaMemcpyHostToDevice),
                       "init SigmaOld"));
  std::vector<double> sc(tups::S_COUNT, 0.0);
  TRY(tups::cuda_check(ctx, cudaMemcpy(s.scal, sc.data(), sc.size() * sizeof(double), cudaMemcpyHostToDevice),
                       "init scalars"));
  return TUPS_OK;
}

namespace tups {
void destroy_events(tups_ctx* ctx);
}

static void free_all(tups_ctx* ctx) {
  for (auto& g : ctx->graph_exec)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  tups::destroy_events(ctx);
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  if (ctx->join_ev) cudaEventDestroy(ctx->join_ev);
  if (ctx->side_stream) cudaStreamDestroy(ctx->side_stream);
  ctx->fork_ev = ctx->join_ev = nullptr;
  ctx->side_stream = nullptr;
  for (void* p : ctx->allocations) cudaFree(p);
  ctx->allocations.clear();
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  ctx->stream = nullptr;
}

// Slots of rank `rank` of `ntasks` (SRC/parquet_ini.f90:336,
// SRC/preprocessing.f90:95-116): Nb = Nred / ntasks contiguous slots from
// rank * Nb; ntasks must divide Nred.
static int shard_slots(tups_ctx* ctx, int rank, int ntasks) {
  tups_dims& d = ctx->d;
  if (ntasks < 1 || rank < 0 || rank >= ntasks)
    return tups::set_error(ctx, TUPS_ERR_BADARG, "rank must lie in [0, ntasks)");
  if (d.Nred % ntasks != 0)
    return tups::set_error(ctx, TUPS_ERR_BADDIM, "choose the number of tasks such that it divides Nred = " +
                                                    std::to_string(d.Nred));
  d.Nb = d.Nred / ntasks;
  ctx->rank = rank;
  ctx->ntasks = ntasks;
  ctx->slot0 = rank * d.Nb;
  return TUPS_OK;
}

static int ctx_create(const tups_params* p, int device, int rank, int ntasks, tups_ctx** out) {
  if (!p || !out) return TUPS_ERR_BADARG;
  *out = nullptr;
  tups_ctx* ctx = new tups_ctx();
  ctx->p = *p;
  ctx->device = device;
  {
    const char* at = std::getenv("TUPS_AUTOTUNE");
    if (at && at[0] == '0') ctx->autotune = false;
  }
  int rc = build_tables(ctx);
  if (rc == TUPS_OK) rc = shard_slots(ctx, rank, ntasks);
  if (rc == TUPS_OK) rc = tups::cuda_check(ctx, cudaSetDevice(device), "cudaSetDevice");
  if (rc == TUPS_OK)
    rc = tups::cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream");
  if (rc == TUPS_OK) rc = upload_tables(ctx);
  if (rc == TUPS_OK) rc = alloc_state(ctx);
  if (rc == TUPS_OK) rc = init_state(ctx);
  if (rc != TUPS_OK) {
    std::fprintf(stderr, "tups_ctx_create: %s\n", ctx->err.c_str());
    free_all(ctx);
    delete ctx;
    return rc;
  }
  *out = ctx;
  return TUPS_OK;
}

extern "C" int tups_read_lambda(const char* fname_L, int Nf, double* L_d, double* L_m, double* L_s,
                                double* L_t) {
  if (!fname_L || Nf < 2 || Nf % 2) return TUPS_ERR_BADARG;
  std::vector<cplx> L[4];
  const std::string base = trim_name(fname_L);
  int rc = read_lambda_file(nullptr, base + "_ph.init", Nf, L[0], L[1]);
  if (!rc) rc = read_lambda_file(nullptr, base + "_pp.init", Nf, L[2], L[3]);
  if (rc) return rc;
  double* out[4] = {L_d, L_m, L_s, L_t};
  for (int r = 0; r < 4; r++)
    if (out[r]) std::memcpy(out[r], L[r].data(), L[r].size() * sizeof(cplx));
  return TUPS_OK;
}

extern "C" int tups_ctx_create(const tups_params* p, int device, tups_ctx** out) {
  return ctx_create(p, device, 0, 1, out);
}

extern "C" int tups_ctx_create_sharded(const tups_params* p, int device, int rank, int ntasks, tups_ctx** out) {
  return ctx_create(p, device, rank, ntasks, out);
}

extern "C" int tups_set_exchange(tups_ctx* ctx, tups_exchange_fn fn, void* user) {
  if (!ctx) return TUPS_ERR_BADARG;
  ctx->xfn = fn;
  ctx->xuser = user;
  return TUPS_OK;
}

extern "C" int tups_get_shard(const tups_ctx* ctx, int* rank, int* ntasks, int* slot0) {
  if (!ctx) return TUPS_ERR_BADARG;
  if (rank) *rank = ctx->rank;
  if (ntasks) *ntasks = ctx->ntasks;
  if (slot0) *slot0 = ctx->slot0;
  return TUPS_OK;
}

extern "C" int tups_ctx_destroy(tups_ctx* ctx) {
  if (!ctx) return TUPS_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_all(ctx);
  delete ctx;
  return TUPS_OK;
}

extern "C" int tups_host_tables(const tups_params* p, tups_dims* d, double* FF, double* FF_inv, int* signs,
                                int* reps, int* lsym, double* lfac, int* ibz) {
  if (!p) return TUPS_ERR_BADARG;
  tups_ctx tmp;
  tmp.p = *p;
  int rc = build_tables(&tmp);
  if (rc != TUPS_OK) {
    std::fprintf(stderr, "tups_host_tables: %s\n", tmp.err.c_str());
    return rc;
  }
  if (d) *d = tmp.d;
  return tups_get_tables(&tmp, FF, FF_inv, signs, reps, lsym, lfac, ibz);
}

extern "C" int tups_get_dims(const tups_ctx* ctx, tups_dims* out) {
  if (!ctx || !out) return TUPS_ERR_BADARG;
  *out = ctx->d;
  return TUPS_OK;
}

extern "C" const char* tups_last_error(const tups_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

extern "C" const char* tups_strerror(int status) {
  switch (status) {
    case TUPS_OK: return "ok";
    case TUPS_ERR_CUDA: return "CUDA runtime error";
    case TUPS_ERR_OOM: return "device out of memory";
    case TUPS_ERR_MU_NOCONV: return "chemical potential bisection did not converge";
    case TUPS_ERR_NAN: return "NaN or Inf in the self-energy or a vertex";
    case TUPS_ERR_TIMEOUT: return "bounded device wait ran out";
    case TUPS_ERR_BADDIM: return "unsupported sizes";
    case TUPS_ERR_BADARG: return "bad argument";
    case TUPS_ERR_IO: return "input file unreadable or malformed";
    case TUPS_ERR_STATE: return "call order violated";
    case TUPS_ERR_COMM: return "exchange between ranks failed";
    default: return "unknown status";
  }
}

extern "C" long long tups_kernel_launches(const tups_ctx* ctx) { return ctx ? ctx->launches : 0; }

extern "C" int tups_get_tables(tups_ctx* ctx, double* FF, double* FF_inv, int* signs, int* reps, int* lsym,
                               double* lfac, int* ibz) {
  if (!ctx) return TUPS_ERR_BADARG;
  if (FF) std::memcpy(FF, ctx->FF.data(), ctx->FF.size() * sizeof(double));
  if (FF_inv) std::memcpy(FF_inv, ctx->FF_inv.data(), ctx->FF_inv.size() * sizeof(double));
  if (signs) std::memcpy(signs, ctx->signs.data(), ctx->signs.size() * sizeof(int));
  if (reps) std::memcpy(reps, ctx->reps.data(), ctx->reps.size() * sizeof(int));
  if (lsym)
    for (size_t i = 0; i < ctx->lsym.size(); i++) lsym[i] = ctx->lsym[i] + 1;
  if (lfac) std::memcpy(lfac, ctx->lfac.data(), ctx->lfac.size() * sizeof(double));
  if (ibz) std::memcpy(ibz, ctx->ibz.data(), ctx->ibz.size() * sizeof(int));
  return TUPS_OK;
}
