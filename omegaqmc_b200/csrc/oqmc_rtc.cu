// Per-system kernel specialisation.
//
// oqmc_specialize() writes a basis policy for the context's molecule as
// straight-line CUDA: one displacement per nucleus, every exponential of every
// exponent group, the contraction sums and the MO accumulation with the
// exponents, normalised contraction coefficients and MO coefficients as
// literals (MO coefficients at round-off level dropped, see Gen::keep).
// NVRTC compiles the move and
// local-energy kernels with that policy for sm_100a and the driver API loads
// them; the sweep entry points then launch these instead of the table-driven
// kernels.  NVRTC and the driver library are opened with dlopen, so the
// library loads (and runs its table-driven kernels) where NVRTC is absent.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <dlfcn.h>
#include <mutex>
#include <string>
#include <vector>
#include <cuda.h>
#include <cuda_runtime.h>
#include <nvrtc.h>

#include "oqmc_rtc.h"
#include "oqmc_rtc_src.inc"   // generated: the kernel headers as strings

namespace {

struct Api {
  bool ok = false;
  std::string err;
  nvrtcResult (*CreateProgram)(nvrtcProgram*, const char*, const char*, int, const char* const*,
                               const char* const*);
  nvrtcResult (*AddNameExpression)(nvrtcProgram, const char*);
  nvrtcResult (*CompileProgram)(nvrtcProgram, int, const char* const*);
  nvrtcResult (*GetProgramLogSize)(nvrtcProgram, size_t*);
  nvrtcResult (*GetProgramLog)(nvrtcProgram, char*);
  nvrtcResult (*GetCUBINSize)(nvrtcProgram, size_t*);
  nvrtcResult (*GetCUBIN)(nvrtcProgram, char*);
  nvrtcResult (*GetLoweredName)(nvrtcProgram, const char*, const char**);
  nvrtcResult (*DestroyProgram)(nvrtcProgram*);
  CUresult (*ModuleLoadData)(CUmodule*, const void*);
  CUresult (*ModuleGetFunction)(CUfunction*, CUmodule, const char*);
  CUresult (*ModuleUnload)(CUmodule);
  CUresult (*FuncSetAttribute)(CUfunction, CUfunction_attribute, int);
  CUresult (*LaunchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned,
                           unsigned, unsigned, CUstream, void**, void**);
  CUresult (*Occupancy)(int*, CUfunction, int, size_t);
  CUresult (*FuncGetAttribute)(int*, CUfunction_attribute, CUfunction);
};

Api g_api;
std::once_flag g_api_once;

template <typename F>
bool sym(void* h, const char* name, F& f) {
  f = reinterpret_cast<F>(dlsym(h, name));
  return f != nullptr;
}

void load_api() {
  const char* nv_names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12",
                            "/usr/local/cuda/lib64/libnvrtc.so"};
  void* nv = nullptr;
  for (const char* n : nv_names)
    if ((nv = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
  void* cu = dlopen("libcuda.so.1", RTLD_NOW | RTLD_LOCAL);
  if (!nv || !cu) {
    g_api.err = !nv ? "NVRTC (libnvrtc.so.12) not found" : "libcuda.so.1 not found";
    return;
  }
  Api& a = g_api;
  bool ok = sym(nv, "nvrtcCreateProgram", a.CreateProgram) &&
            sym(nv, "nvrtcAddNameExpression", a.AddNameExpression) &&
            sym(nv, "nvrtcCompileProgram", a.CompileProgram) &&
            sym(nv, "nvrtcGetProgramLogSize", a.GetProgramLogSize) &&
            sym(nv, "nvrtcGetProgramLog", a.GetProgramLog) &&
            sym(nv, "nvrtcGetCUBINSize", a.GetCUBINSize) &&
            sym(nv, "nvrtcGetCUBIN", a.GetCUBIN) &&
            sym(nv, "nvrtcGetLoweredName", a.GetLoweredName) &&
            sym(nv, "nvrtcDestroyProgram", a.DestroyProgram) &&
            sym(cu, "cuModuleLoadData", a.ModuleLoadData) &&
            sym(cu, "cuModuleGetFunction", a.ModuleGetFunction) &&
            sym(cu, "cuModuleUnload", a.ModuleUnload) &&
            sym(cu, "cuFuncSetAttribute", a.FuncSetAttribute) &&
            sym(cu, "cuLaunchKernel", a.LaunchKernel) &&
            sym(cu, "cuOccupancyMaxActiveBlocksPerMultiprocessor", a.Occupancy) &&
            sym(cu, "cuFuncGetAttribute", a.FuncGetAttribute);
  if (!ok) {
    a.err = "missing NVRTC or driver symbol";
    return;
  }
  a.ok = true;
}

// ---------------------------------------------------------------------------
// source generation
// ---------------------------------------------------------------------------
struct Gen {
  const OqSystem& S;
  const OqSplit& SP;
  const double* C;     // nbf x nocc
  int nocc;
  std::string o;
  bool contract = false;   // VGL contracted with an inverse column (mo_vgl_contract)
  std::vector<double> cmax;  // largest |C[.][m]| of each orbital
  void add(const std::string& s) { o += s; }

  // Whether C[ao][m] enters the generated code.  An orbital of a molecule
  // with point-group symmetry has exact zeros on the AOs of other irreducible
  // representations, which an eigensolver returns as round-off (1e-15 of the
  // orbital's largest coefficient; half of the H2O coefficients).  Terms
  // below 1e-12 of that largest coefficient change an orbital value by less
  // than 1e-12 of its scale, far below the FP64 parity tolerance, so they
  // are left out of the straight-line code.
  bool keep(int ao, int m) {
    if (cmax.empty()) {
      cmax.assign(nocc, 0.0);
      for (int mu = 0; mu < S.nbf; ++mu)
        for (int k = 0; k < nocc; ++k) cmax[k] = std::max(cmax[k], std::fabs(C[mu * nocc + k]));
    }
    const double c = std::fabs(C[ao * nocc + m]);
    return c != 0.0 && c > 1e-12 * cmax[m];
  }

  static std::string num(double v) {
    char b[40];
    snprintf(b, sizeof b, "%.17g", v);
    std::string s(b);
    if (s.find_first_of(".eEn") == std::string::npos) s += ".0";
    return s;
  }

  // Primitive p of group g is tight when its own split radius 25 / alpha
  // is within the group's (the largest over its tight primitives).
  bool tight(int g, int p) const {
    return SP.r2[g] > 0.0 && S.alpha[S.g_off[g] + p] * SP.r2[g] >= 25.0 * (1.0 - 1e-12);
  }

  // declare R<k> (and Rp<k>, Rl<k>) of type ty and accumulate group g's
  // primitives (sel 0: all, 1: tight only, 2: all but the tight ones).  With
  // e_p = exp(-a_p r^2): R = sum n_p e_p, R'/r = sum (-2 a_p n_p) e_p and
  // R'' + 2 R'/r = r^2 sum (4 a_p^2 n_p) e_p + 3 R'/r, the per-primitive
  // constants folded on the host.
  void radial(int g, bool vgl, const std::string& ty, const char* r2, int sel = 0,
              bool tight_arg = false) {
    const int np = S.g_n[g], nc = S.g_ncol[g], off = S.g_off[g], sh0 = S.g_shell0[g];
    for (int k = 0; k < nc; ++k) {
      const std::string ks = std::to_string(k);
      add("      " + ty + " R" + ks + " = 0");
      if (vgl) add(", Rp" + ks + " = 0, Rl" + ks + ", Ra" + ks + " = 0");
      add(";\n");
    }
    for (int p = 0; p < np; ++p) {
      if ((sel == 1 && !tight(g, p)) || (sel == 2 && tight(g, p))) continue;
      const double a = S.alpha[off + p];
      if (tight_arg && tight(g, p))   // FP64 argument, see oq_exp_tight
        add("      { const " + ty + " e = oq_exp_tight<" + ty + ">(" + num(a) + ", " +
            num(a * 1.4426950408889634) + ", r2d);\n");
      else if (ty == "double")
        add("      { const double e = exp(-((double)" + num(a) + ") * " + r2 + ");\n");
      else   // a and a log2(e) folded here, see oq_exp_neg
        add("      { const T e = oq_exp_neg<T>((T)" + num(a) + ", (T)" +
            num(a * 1.4426950408889634) + ", " + r2 + ");\n");
      for (int k = 0; k < nc; ++k) {
        const double n = S.norm[S.s_norm[sh0 + k] + p];
        const std::string ks = std::to_string(k);
        add("        R" + ks + " += ((" + ty + ")" + num(n) + ") * e;");
        if (vgl)
          add(" Rp" + ks + " += ((" + ty + ")" + num(-2.0 * a * n) + ") * e; Ra" + ks +
              " += ((" + ty + ")" + num(4.0 * a * a * n) + ") * e;");
        add("\n");
      }
      add("      }\n");
    }
    if (vgl)
      for (int k = 0; k < nc; ++k) {
        const std::string ks = std::to_string(k);
        add("      Rl" + ks + " = " + r2 + " * Ra" + ks + " + (" + ty + ")3 * Rp" + ks + ";\n");
      }
  }

  // ca = sum_m C[ao][m] ac[m] over the kept coefficients ("" when none)
  std::string ca_expr(int ao) {
    std::string ca;
    for (int m = 0; m < nocc; ++m) {
      if (!keep(ao, m)) continue;
      ca += std::string(ca.empty() ? "" : " + ") + "(T)(" + num(C[ao * nocc + m]) + ") * ac[" +
            std::to_string(m) + "]";
    }
    return ca;
  }

  // accumulate one AO into the MOs (value expression v; grad g[3], lap l)
  void accum(int ao, const std::string& v, const std::string* g, const std::string* l) {
    for (int m = 0; m < nocc; ++m) {
      const double c = C[ao * nocc + m];
      if (!keep(ao, m)) continue;
      const std::string cl = "(T)(" + num(c) + ")", ms = std::to_string(m);
      add("      mv[" + ms + "] += " + cl + " * " + v + ";\n");
      if (g) {
        add("      mg[" + ms + "][0] += " + cl + " * " + g[0] + "; mg[" + ms + "][1] += " + cl +
            " * " + g[1] + "; mg[" + ms + "][2] += " + cl + " * " + g[2] + ";\n");
        add("      ml[" + ms + "] += " + cl + " * " + *l + ";\n");
      }
    }
  }

  // angular factors of column k of group g; radial names R, Rp, Rl
  void angular(int g, int k, bool vgl, const std::string& R, const std::string& Rp,
               const std::string& Rl) {
    const int am = S.g_am[g];
    const int ao = S.s_ao[S.g_shell0[g] + k];
    if (contract) {
      angular_contract(am, ao, R, Rp, Rl);
      return;
    }
    add("    {\n");
    if (am == 0) {
      if (!vgl) {
        accum(ao, R, nullptr, nullptr);
      } else {
        std::string gg[3] = {"(" + Rp + " * dx)", "(" + Rp + " * dy)", "(" + Rp + " * dz)"};
        accum(ao, R, gg, &Rl);
      }
    } else {
      if (vgl) add("      const T lfac = " + Rl + " + (T)" + std::to_string(2 * am) + " * " + Rp + ";\n");
      if (am == 2) add("      T Y[5], dY[5][3]; oq_harm_d<T>(dx, dy, dz, Y, dY);\n");
      for (int c = 0; c < 2 * am + 1; ++c) {
        const std::string cs = std::to_string(c);
        std::string Y, d0, d1, d2;
        if (am == 1) {
          Y = c == 0 ? "dx" : c == 1 ? "dy" : "dz";
          d0 = c == 0 ? "(T)1" : ""; d1 = c == 1 ? "(T)1" : ""; d2 = c == 2 ? "(T)1" : "";
        } else if (am == 2) {
          Y = "Y[" + cs + "]"; d0 = "dY[" + cs + "][0]"; d1 = "dY[" + cs + "][1]"; d2 = "dY[" + cs + "][2]";
        } else {
          add("      T Y" + cs + ", dY" + cs + "[3]; oq_harm_table<T>(S.harm, " + std::to_string(am) +
              ", " + cs + ", dx, dy, dz, Y" + cs + ", dY" + cs + ");\n");
          Y = "Y" + cs; d0 = "dY" + cs + "[0]"; d1 = "dY" + cs + "[1]"; d2 = "dY" + cs + "[2]";
        }
        if (!vgl) {
          accum(ao + c, "(" + R + " * " + Y + ")", nullptr, nullptr);
        } else {
          // (a p function's gradient has R in one component only: no R * 0 terms)
          auto term = [&](const char* dc, const std::string& dy) {
            return "(" + Rp + " * " + dc + " * " + Y + (dy.empty() ? "" : " + " + R + " * " + dy) +
                   ")";
          };
          std::string gg[3] = {term("dx", d0), term("dy", d1), term("dz", d2)};
          std::string ll = "(lfac * " + Y + ")";
          accum(ao + c, "(" + R + " * " + Y + ")", gg, &ll);
        }
      }
    }
    add("    }\n");
  }

  // Contracted VGL of one shell column (angular momentum am, AOs ao ...
  // ao + 2 am): with c_q = ca of AO q, A = sum_q c_q Y_q and G = sum_q c_q
  // grad Y_q, the column adds Rp A d to the gradient (summed per nucleus in
  // sR, multiplied by d once), R G to the gradient and (Rl + 2 am Rp) A to
  // the Laplacian (solid harmonics have no Laplacian of their own).  Columns
  // whose AOs no kept coefficient reaches are left out.
  void angular_contract(int am, int ao, const std::string& R, const std::string& Rp,
                        const std::string& Rl) {
    const int nq = 2 * am + 1;
    std::vector<std::string> cq(nq);
    bool any = false;
    for (int q = 0; q < nq; ++q) {
      cq[q] = ca_expr(ao + q);
      any = any || !cq[q].empty();
    }
    if (!any) return;
    add("    {\n");
    if (am == 0) {
      add("      const T c0 = " + cq[0] + ";\n      sR += " + Rp + " * c0; lp += " + Rl +
          " * c0;\n    }\n");
      return;
    }
    for (int q = 0; q < nq; ++q)
      if (!cq[q].empty()) add("      const T c" + std::to_string(q) + " = " + cq[q] + ";\n");
    std::string A, G[3];
    auto plus = [](std::string& acc, const std::string& t) {
      acc += (acc.empty() ? "" : " + ") + t;
    };
    if (am == 1) {
      const char* dn[3] = {"dx", "dy", "dz"};
      for (int q = 0; q < 3; ++q)
        if (!cq[q].empty()) {
          plus(A, "c" + std::to_string(q) + " * " + dn[q]);
          G[q] = "c" + std::to_string(q);
        }
    } else {
      if (am == 2) add("      T Y[5], dY[5][3]; oq_harm_d<T>(dx, dy, dz, Y, dY);\n");
      for (int q = 0; q < nq; ++q) {
        if (cq[q].empty()) continue;
        const std::string qs = std::to_string(q), cn = "c" + qs;
        std::string Y, dY;
        if (am == 2) {
          Y = "Y[" + qs + "]";
          dY = "dY[" + qs + "]";
        } else {
          add("      T Y" + qs + ", dY" + qs + "[3]; oq_harm_table<T>(S.harm, " +
              std::to_string(am) + ", " + qs + ", dx, dy, dz, Y" + qs + ", dY" + qs + ");\n");
          Y = "Y" + qs;
          dY = "dY" + qs;
        }
        plus(A, cn + " * " + Y);
        for (int j = 0; j < 3; ++j) plus(G[j], cn + " * " + dY + "[" + std::to_string(j) + "]");
      }
    }
    add("      const T A = " + A + ";\n      sR += " + Rp + " * A; lp += (" + Rl + " + (T)" +
        std::to_string(2 * am) + " * " + Rp + ") * A;\n");
    const char* gn[3] = {"gx", "gy", "gz"};
    for (int j = 0; j < 3; ++j)
      if (!G[j].empty()) add("      " + std::string(gn[j]) + " += " + R + " * (" + G[j] + ");\n");
    add("    }\n");
  }

  void body(bool vgl) {
    if (contract) add("  gx = (T)0; gy = (T)0; gz = (T)0; lp = (T)0;\n");
    for (int m = 0; m < nocc && !contract; ++m) {
      const std::string ms = std::to_string(m);
      add("  mv[" + ms + "] = (T)0;");
      if (vgl)
        add(" mg[" + ms + "][0] = (T)0; mg[" + ms + "][1] = (T)0; mg[" + ms + "][2] = (T)0; ml[" +
            ms + "] = (T)0;");
      add("\n");
    }
    for (int ia = 0; ia < S.natm; ++ia) {
      bool any = false;
      for (int g = 0; g < S.ngroup; ++g) any = any || S.g_iat[g] == ia;
      if (!any) continue;
      add("  {\n  const double dxd = x - (" + num(S.nuc[ia][0]) + "), dyd = y - (" +
          num(S.nuc[ia][1]) + "), dzd = z - (" + num(S.nuc[ia][2]) + ");\n"
          "  const double r2d = dxd * dxd + dyd * dyd + dzd * dzd;\n"
          "  const T dx = (T)dxd, dy = (T)dyd, dz = (T)dzd, r2 = (T)r2d;\n  (void)r2;\n");
      if (contract) add("  T sR = (T)0;\n");
      for (int g = 0; g < S.ngroup; ++g) {
        if (S.g_iat[g] != ia) continue;
        const int nc = S.g_ncol[g], sh0 = S.g_shell0[g];
        const bool s_shell = S.g_am[g] == 0;
        add("  {\n");
        if (!vgl) {
          radial(g, false, "T", "r2");
          for (int k = 0; k < nc; ++k)
            if (s_shell && S.s_cusp[sh0 + k])
              add("    R" + std::to_string(k) + " = (T)oq_cusp_val(S, " + std::to_string(ia) +
                  ", sqrt(r2d), (double)R" + std::to_string(k) + ");\n");
          for (int k = 0; k < nc; ++k) {
            const std::string ks = std::to_string(k);
            angular(g, k, false, "R" + ks, "", "");
          }
        } else {
          // Radial factors: cusp groups in FP64; the tight exponents of a
          // split group with FP64 arguments; everything else in the working
          // precision.
          bool cusp = false;
          for (int k = 0; k < nc; ++k) cusp = cusp || (s_shell && S.s_cusp[sh0 + k]);
          const bool split = SP.r2[g] > 0.0;
          for (int k = 0; k < nc; ++k) {
            const std::string ks = std::to_string(k);
            add("    T RT" + ks + ", RpT" + ks + ", RlT" + ks + ";\n");
          }
          auto fp64_inline = [&]() {
            add("      {\n");
            radial(g, true, "double", "r2d");
            for (int k = 0; k < nc; ++k) {
              const std::string ks = std::to_string(k);
              if (s_shell && S.s_cusp[sh0 + k])
                add("      oq_cusp_vgl(S, " + std::to_string(ia) + ", sqrt(r2d), R" + ks + ", Rp" +
                    ks + ", Rl" + ks + ");\n");
              add("      RT" + ks + " = (T)R" + ks + "; RpT" + ks + " = (T)Rp" + ks + "; RlT" + ks +
                  " = (T)Rl" + ks + ";\n");
            }
            add("      }\n");
          };
          auto working = [&]() {
            add("      {\n");
            radial(g, true, "T", "r2");
            for (int k = 0; k < nc; ++k) {
              const std::string ks = std::to_string(k);
              add("      RT" + ks + " = R" + ks + "; RpT" + ks + " = Rp" + ks + "; RlT" + ks +
                  " = Rl" + ks + ";\n");
            }
            add("      }\n");
          };
          if (cusp) {
            fp64_inline();
          } else if (split) {
            // the tight exponents with FP64 arguments (oq_exp_tight), every
            // lane and every exponent of the group in the working precision
            add("      {\n");
            radial(g, true, "T", "r2", 0, true);
            for (int k = 0; k < nc; ++k) {
              const std::string ks = std::to_string(k);
              add("      RT" + ks + " = R" + ks + "; RpT" + ks + " = Rp" + ks + "; RlT" + ks +
                  " = Rl" + ks + ";\n");
            }
            add("      }\n");
          } else {
            working();
          }
          for (int k = 0; k < nc; ++k) {
            const std::string ks = std::to_string(k);
            angular(g, k, true, "RT" + ks, "RpT" + ks, "RlT" + ks);
          }
        }
        add("  }\n");
      }
      if (contract) add("  gx += sR * dx; gy += sR * dy; gz += sR * dz;\n");
      add("  }\n");
    }
  }
};

// The basis policy of one system as a struct named `name`.
std::string generate_basis(const OqSystem& S, const OqSplit& SP, const double* C, int nocc,
                           const std::string& name) {
  std::string src = "struct " + name + " {\n";
  {
    Gen g{S, SP, C, nocc, ""};
    g.body(false);
    src += "  template <typename T, typename TC>\n"
           "  __device__ static __forceinline__ void mo_val(const OqSystem& S, const OqSplit& SP,\n"
           "      const TC* __restrict__ C, double x, double y, double z, T* mv) {\n"
           "  (void)SP; (void)C;\n";
    src += g.o + "  }\n\n";
  }
  {
    Gen g{S, SP, C, nocc, ""};
    g.body(true);
    std::string b = g.o;
    src += "  template <typename T, typename TC>\n"
           "  __device__ static __forceinline__ void mo_vgl(const OqSystem& S, const OqSplit& SP,\n"
           "      const TC* __restrict__ C, double x, double y, double z, T* mv, T (*mg)[3],\n"
           "      T* ml) {\n  (void)SP; (void)C;\n";
    src += b + "  }\n";
  }
  {
    Gen g{S, SP, C, nocc, ""};
    g.contract = true;
    g.body(true);
    src += "\n  // gradient and Laplacian of sum_m ac[m] phi_m (the Slater part of the local\n"
           "  // energy with ac a column of the inverse)\n"
           "  template <typename T, typename TC>\n"
           "  __device__ static __forceinline__ void mo_vgl_contract(const OqSystem& S,\n"
           "      const OqSplit& SP, const TC* __restrict__ C, double x, double y, double z,\n"
           "      const T* ac, T& gx, T& gy, T& gz, T& lp) {\n  (void)SP; (void)C;\n";
    src += g.o + "  }\n";
  }
  src += "};\n";
  return src;
}

std::string generate(const OqSystem& S, const OqSplit& SP, const double* C, int nocc) {
  return "#include \"oqmc_sweep.cuh\"\n\n" + generate_basis(S, SP, C, nocc, "OqSpecBasis");
}

}  // namespace

std::string oq_spec_basis_source(const OqSystem& S, const OqSplit& SP, const double* C, int nocc,
                                 const std::string& name) {
  return generate_basis(S, SP, C, nocc, name);
}

int oq_rtc_available(std::string* err) {
  std::call_once(g_api_once, load_api);
  if (!g_api.ok && err) *err = g_api.err;
  return g_api.ok ? 1 : 0;
}

int oq_rtc_compile(const std::string& src, const std::vector<std::string>& names,
                   std::vector<char>* cubin, std::vector<std::string>* lowered,
                   std::string* err) {
  std::call_once(g_api_once, load_api);
  if (!g_api.ok) {
    *err = g_api.err;
    return -1;
  }
  const Api& A = g_api;
  std::vector<const char*> hdr_src, hdr_name;
  for (int i = 0; i < kOqRtcCount; ++i) {
    hdr_src.push_back(kOqRtcSrcs[i]);
    hdr_name.push_back(kOqRtcNames[i]);
  }
  nvrtcProgram prog;
  if (A.CreateProgram(&prog, src.c_str(), "oqmc_rtc.cu", kOqRtcCount, hdr_src.data(),
                      hdr_name.data()) != NVRTC_SUCCESS) {
    *err = "nvrtcCreateProgram failed";
    return -1;
  }
  for (const std::string& n : names) A.AddNameExpression(prog, n.c_str());
  const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-lineinfo",
                        "--device-as-default-execution-space"};
  const nvrtcResult rc = A.CompileProgram(prog, 4, opts);
  if (rc != NVRTC_SUCCESS) {
    size_t n = 0;
    A.GetProgramLogSize(prog, &n);
    std::string log(n, '\0');
    A.GetProgramLog(prog, &log[0]);
    *err = "NVRTC compile failed: " + log.substr(0, 2000);
    A.DestroyProgram(&prog);
    return -1;
  }
  size_t nb = 0;
  A.GetCUBINSize(prog, &nb);
  cubin->resize(nb);
  A.GetCUBIN(prog, cubin->data());
  lowered->assign(names.size(), "");
  for (size_t i = 0; i < names.size(); ++i) {
    const char* ln = nullptr;
    A.GetLoweredName(prog, names[i].c_str(), &ln);
    (*lowered)[i] = ln ? ln : "";
  }
  A.DestroyProgram(&prog);
  return 0;
}

int oq_rtc_load(const std::vector<char>& cubin, const std::vector<std::string>& lowered,
                void** mod_out, std::vector<void*>* fns, std::string* err) {
  const Api& A = g_api;
  CUmodule mod = nullptr;
  if (A.ModuleLoadData(&mod, cubin.data()) != CUDA_SUCCESS) {
    *err = "cuModuleLoadData failed";
    return -1;
  }
  fns->assign(lowered.size(), nullptr);
  for (size_t i = 0; i < lowered.size(); ++i) {
    CUfunction f = nullptr;
    if (A.ModuleGetFunction(&f, mod, lowered[i].c_str()) != CUDA_SUCCESS) {
      A.ModuleUnload(mod);
      *err = "cuModuleGetFunction failed for " + lowered[i];
      return -1;
    }
    A.FuncSetAttribute(f, CU_FUNC_ATTRIBUTE_PREFERRED_SHARED_MEMORY_CARVEOUT, 100);
    (*fns)[i] = (void*)f;
  }
  *mod_out = (void*)mod;
  return 0;
}

int oq_rtc_build(const std::string& src, const std::vector<std::string>& names, void** mod_out,
                 std::vector<void*>* fns, std::string* err) {
  std::vector<char> cubin;
  std::vector<std::string> lowered;
  if (oq_rtc_compile(src, names, &cubin, &lowered, err) != 0) return -1;
  return oq_rtc_load(cubin, lowered, mod_out, fns, err);
}

void oq_rtc_unload(void* mod) {
  if (g_api.ok && mod) g_api.ModuleUnload((CUmodule)mod);
}

int oq_rtc_launch(void* fn, dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                  void** args) {
  const Api& A = g_api;
  CUfunction f = (CUfunction)fn;
  if (smem > 48 * 1024 &&
      A.FuncSetAttribute(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem) !=
          CUDA_SUCCESS)
    return -1;
  return A.LaunchKernel(f, grid.x, grid.y, grid.z, block.x, block.y, block.z, (unsigned)smem,
                        (CUstream)stream, args, nullptr) == CUDA_SUCCESS
             ? 0
             : -1;
}

int oq_rtc_occupancy(void* fn, int block, size_t smem, int* nblk) {
  const Api& A = g_api;
  CUfunction f = (CUfunction)fn;
  if (smem > 48 * 1024 &&
      A.FuncSetAttribute(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem) !=
          CUDA_SUCCESS) {
    *nblk = 0;
    return 0;
  }
  return A.Occupancy(nblk, f, block, smem) == CUDA_SUCCESS ? 0 : -1;
}

int oq_rtc_regs(void* fn) {
  int r = -1;
  g_api.FuncGetAttribute(&r, CU_FUNC_ATTRIBUTE_NUM_REGS, (CUfunction)fn);
  return r;
}

int oq_rtc_local_bytes(void* fn) {
  int r = -1;
  g_api.FuncGetAttribute(&r, CU_FUNC_ATTRIBUTE_LOCAL_SIZE_BYTES, (CUfunction)fn);
  return r;
}

struct OqSpecModule {
  CUmodule mod = nullptr;
  // moves fixed-width d/f, eloc d/f, moves nucleus-scaled d/f
  CUfunction fn[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

int oq_spec_build(const OqSystem& S, const OqSplit& SP, const double* C, int nocc,
                  OqSpecModule** out, std::string* err) {
  std::vector<std::string> names;
  const char* forms[6] = {"k_moves<%d, double, double, 0, OqSpecBasis>",
                          "k_moves<%d, float, float, 0, OqSpecBasis>",
                          "k_eloc<%d, double, double, OqSpecBasis>",
                          "k_eloc<%d, float, float, OqSpecBasis>",
                          "k_moves<%d, double, double, 1, OqSpecBasis>",
                          "k_moves<%d, float, float, 1, OqSpecBasis>"};
  for (const char* f : forms) {
    char b[128];
    snprintf(b, sizeof b, f, nocc);
    names.push_back(b);
  }
  void* mod = nullptr;
  std::vector<void*> fns;
  if (oq_rtc_build(generate(S, SP, C, nocc), names, &mod, &fns, err) != 0) return -1;
  OqSpecModule* m = new OqSpecModule();
  m->mod = (CUmodule)mod;
  for (int i = 0; i < 6; ++i) m->fn[i] = (CUfunction)fns[i];
  *out = m;
  return 0;
}

void oq_spec_destroy(OqSpecModule* m) {
  if (!m) return;
  if (g_api.ok && m->mod) g_api.ModuleUnload(m->mod);
  delete m;
}

void* oq_spec_function(OqSpecModule* m, int which) {
  return (m && which >= 0 && which < 6) ? (void*)m->fn[which] : nullptr;
}

int oq_spec_launch(OqSpecModule* m, int which, dim3 grid, dim3 block, size_t smem,
                   cudaStream_t stream, void** args) {
  const Api& A = g_api;
  CUfunction f = m->fn[which];
  if (smem > 48 * 1024 &&
      A.FuncSetAttribute(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem) !=
          CUDA_SUCCESS)
    return -1;
  return A.LaunchKernel(f, grid.x, grid.y, grid.z, block.x, block.y, block.z, (unsigned)smem,
                        (CUstream)stream, args, nullptr) == CUDA_SUCCESS
             ? 0
             : -1;
}

std::string oq_spec_source(const OqSystem& S, const OqSplit& SP, const double* C, int nocc) {
  return generate(S, SP, C, nocc);
}
