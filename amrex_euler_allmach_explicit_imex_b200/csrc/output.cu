// Output writers of a run (io/output_cases.hpp): the final CSVs of the report
// problems (Gresho, Toro, Riemann quadrant, advection blob), and the
// shock-density-bubble snapshots, metrics and summary.
//
// B200 formulation: the per-cell columns (primitives, exact or initial states,
// internal energy, schlieren) are computed on the device in the reference's
// arithmetic (this file is built with -fmad=false and IEEE division and square
// root), the bubble metrics are one device reduction, and only the columns
// cross to the host.  Rows are formatted with %.17g (the reference's
// std::setprecision(17)) by all host threads, each taking a contiguous block
// of rows, and written in order.  A snapshot can be written asynchronously:
// the column kernel runs on the context's stream, the copy to pinned memory on
// a side stream, and a writer thread formats the file while stepping goes on
// (two slots; a third request waits for the oldest).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <limits>
#include <string>
#include <thread>
#include <vector>

#define ECG_NS ecg_out
#include "stencil.cuh"
#include "ctx.h"

namespace ecg_out {

enum OutKind : int { K_GRESHO = 0, K_TORO = 1, K_QUADRANT = 2, K_BLOB = 3, K_BUBBLE = 4 };
constexpr int kCols = 8;  // planes of the column buffer
constexpr int kMetricBlocks = 296;
constexpr int kNT = 256;
constexpr double kBubbleThreshold = 0.55;  // density_bubble_area_threshold (io/output_cases.hpp:253)

// Per-cell columns, planes of n doubles: rho, u, v, p (to_primitive), then
// by kind: the exact Gresho / blob state or the initial quadrant state
// (4..7); for the bubble, internal energy and schlieren (4, 5).
__global__ void __launch_bounds__(kNT) fields_kernel(const EcgFvParams P, const EcgProblem pr,
                                                     const double* __restrict__ u, int kind, double time,
                                                     double* __restrict__ out)
{
  const int nx = P.g.nx;
  const long long n = static_cast<long long>(nx) * P.g.ny;
  const double dx = P.g.dx, dy = P.g.dy;
  for (long long r = blockIdx.x * static_cast<long long>(kNT) + threadIdx.x; r < n;
       r += static_cast<long long>(gridDim.x) * kNT) {
    const int j = static_cast<int>(r / nx), i = static_cast<int>(r - static_cast<long long>(j) * nx);
    const double x = P.g.plo_x + (static_cast<double>(i) + 0.5) * dx;
    const double y = P.g.plo_y + (static_cast<double>(j) + 0.5) * dy;
    const Cons c = load_cell(P, u, i, j);
    const Prim q = to_prim(c, P.gamma);
    double col[kCols] = {q.rho, q.u, q.v, q.p, 0.0, 0.0, 0.0, 0.0};
    if (kind == K_GRESHO || kind == K_QUADRANT || kind == K_BLOB) {
      const Prim e = kind == K_GRESHO ? gresho_state(x, y, pr)
                                      : (kind == K_QUADRANT ? quadrant_state(x, y, pr)
                                                            : exact_blob_state(x, y, pr, P.g.plo_x, P.g.plo_y, time));
      col[4] = e.rho;
      col[5] = e.u;
      col[6] = e.v;
      col[7] = e.p;
    } else if (kind == K_BUBBLE) {
      // io/output_cases.hpp:462-471
      const double kinetic = 0.5 * (c.mx * c.mx + c.my * c.my) / c.rho;
      col[4] = c.E - kinetic;
      const double rho_x = (load_cell(P, u, i + 1, j).rho - load_cell(P, u, i - 1, j).rho) / (2.0 * dx);
      const double rho_y = (load_cell(P, u, i, j + 1).rho - load_cell(P, u, i, j - 1).rho) / (2.0 * dy);
      col[5] = sqrt(rho_x * rho_x + rho_y * rho_y);
    }
#pragma unroll
    for (int k = 0; k < kCols; ++k) out[k * n + r] = col[k];
  }
}

// compute_shock_density_bubble_metrics (io/output_cases.hpp:329-403), one
// partial record per block; the host combines the blocks in order.
struct MetricPart {
  double rho_min, rho_max, p_min, p_max, ie_min, area, cx_sum, cy_sum, schlieren;
  long long nonfinite;
};

__global__ void __launch_bounds__(kNT) metrics_kernel(const EcgFvParams P, const double* __restrict__ u,
                                                      MetricPart* __restrict__ part)
{
  const int nx = P.g.nx;
  const long long n = static_cast<long long>(nx) * P.g.ny;
  const double dx = P.g.dx, dy = P.g.dy;
  const double vol = dx * dy;  // cell_volume (core/state_primitives.hpp:3-7)
  const double inf = __builtin_huge_val();
  MetricPart m{inf, -inf, inf, -inf, inf, 0.0, 0.0, 0.0, 0.0, 0};
  for (long long r = blockIdx.x * static_cast<long long>(kNT) + threadIdx.x; r < n;
       r += static_cast<long long>(gridDim.x) * kNT) {
    const int j = static_cast<int>(r / nx), i = static_cast<int>(r - static_cast<long long>(j) * nx);
    const Cons c = load_cell(P, u, i, j);
    const Prim q = to_prim(c, P.gamma);
    const double kinetic = c.rho > 0.0 ? 0.5 * (c.mx * c.mx + c.my * c.my) / c.rho : __longlong_as_double(0x7ff8000000000000LL);
    const double internal = c.E - kinetic;
    const bool bad = !isfinite(c.rho) || !isfinite(c.mx) || !isfinite(c.my) || !isfinite(c.E) || !isfinite(q.p) ||
                     !isfinite(internal);
    if (bad) {
      ++m.nonfinite;
      continue;
    }
    m.rho_min = fmin(m.rho_min, q.rho);
    m.rho_max = fmax(m.rho_max, q.rho);
    m.p_min = fmin(m.p_min, q.p);
    m.p_max = fmax(m.p_max, q.p);
    m.ie_min = fmin(m.ie_min, internal);
    const double rho_x = (load_cell(P, u, i + 1, j).rho - load_cell(P, u, i - 1, j).rho) / (2.0 * dx);
    const double rho_y = (load_cell(P, u, i, j + 1).rho - load_cell(P, u, i, j - 1).rho) / (2.0 * dy);
    const double grad = sqrt(rho_x * rho_x + rho_y * rho_y);
    if (isfinite(grad)) m.schlieren = fmax(m.schlieren, grad);
    if (q.rho < kBubbleThreshold) {
      const double x = P.g.plo_x + (static_cast<double>(i) + 0.5) * dx;
      const double y = P.g.plo_y + (static_cast<double>(j) + 0.5) * dy;
      m.area += vol;
      m.cx_sum += x * vol;
      m.cy_sum += y * vol;
    }
  }
  // block combine in thread order (shared memory, thread 0)
  __shared__ MetricPart sh[kNT];
  sh[threadIdx.x] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    MetricPart b = sh[0];
    for (int t = 1; t < kNT; ++t) {
      const MetricPart& o = sh[t];
      b.rho_min = fmin(b.rho_min, o.rho_min);
      b.rho_max = fmax(b.rho_max, o.rho_max);
      b.p_min = fmin(b.p_min, o.p_min);
      b.p_max = fmax(b.p_max, o.p_max);
      b.ie_min = fmin(b.ie_min, o.ie_min);
      b.area += o.area;
      b.cx_sum += o.cx_sum;
      b.cy_sum += o.cy_sum;
      b.schlieren = fmax(b.schlieren, o.schlieren);
      b.nonfinite += o.nonfinite;
    }
    part[blockIdx.x] = b;
  }
}

}  // namespace ecg_out

// ---- host side ---------------------------------------------------------------------------

namespace {

using ecg_out::kCols;

// Labels of core/config_parse_helpers.hpp:117-196 and the bubble case strings
// of problems/problem_initialization.hpp:37-50 (kept alike: they are columns
// of the files the report scripts read).
const char* method_label(int m) { return m == ECG_METHOD_IMEX ? "imex" : "explicit"; }
const char* riemann_label(int r)
{
  switch (r) {
    case ECG_RIEMANN_RUSANOV:
      return "rusanov";
    case ECG_RIEMANN_LOWMACH_HLLC:
      return "lowmach_hllc";
    case ECG_RIEMANN_XIE_AM_HLLC_P:
      return "xie_am_hllc_p";
    default:
      return "hllc";
  }
}
const char* limiter_label(int l) { return l == ECG_LIMITER_MC ? "mc" : (l == ECG_LIMITER_VANLEER ? "vanleer" : "minmod"); }
const char* kImexForm = "bdltv20_t1_s2_source_map_picard";
const char* kImexPredictorFlux = "bdltv20_pressure_split_lf";
const char* kImexPredictorDissipation = "material";  // the only setting the IMEX method accepts
const char* kBubbleCaseId = "same_gamma_shock_density_bubble_clawpack_style_v1";
const char* kBubbleClaim = "qualitative_project_high_speed_2d_only";
// shock_density_bubble_* (problems/problem_initialization.hpp:2-58)
constexpr double kBubbleShockX = 0.2, kBubbleCx = 0.5, kBubbleCy = 0.0, kBubbleR = 0.2, kBubbleRho = 0.1;
constexpr double kPostShock[4] = {2.8181818181818183, 1.6064386578049976, 0.0, 5.0};

std::string bubble_scheme_name(const ecg_run_config& c)
{
  if (c.method == ECG_METHOD_IMEX) return "imex_t1s2_bdltv20_ideal_gas";
  if (c.riemann == ECG_RIEMANN_XIE_AM_HLLC_P) return "explicit_o2_low_mach_corrected_hllc_p";
  if (c.riemann == ECG_RIEMANN_HLLC) return "explicit_o2_hllc";
  return std::string("explicit_o") + std::to_string(c.spatial_order) + "_" + riemann_label(c.riemann);
}

// csv_escape (io/output_cases.hpp:236-251)
std::string csv_escape(const std::string& v)
{
  if (v.find_first_of(",\"\n") == std::string::npos) return v;
  std::string e = "\"";
  for (const char ch : v) e += ch == '"' ? std::string("\"\"") : std::string(1, ch);
  return e + "\"";
}

// Row text in the reference's stream format.
struct Row {
  std::string& s;
  char b[40];
  Row& d(double v)
  {
    std::snprintf(b, sizeof(b), "%.17g", v);
    s += b;
    return *this;
  }
  Row& i(long long v)
  {
    std::snprintf(b, sizeof(b), "%lld", v);
    s += b;
    return *this;
  }
  Row& t(const char* v)
  {
    s += v;
    return *this;
  }
  Row& c()
  {
    s += ',';
    return *this;
  }
};

// Formats rows [0, n) with fmt(row, text) on all host threads (contiguous
// blocks of rows) and writes header + rows in order.  false on an I/O error.
template <class F>
bool write_rows(const std::string& path, const std::string& header, long long n, F fmt)
{
  std::FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  bool ok = std::fwrite(header.data(), 1, header.size(), f) == header.size();
  unsigned hw = std::thread::hardware_concurrency();
  const int nt = static_cast<int>(std::max(1u, std::min(hw ? hw : 1u, 64u)));
  const long long block = 65536;  // rows per formatting batch
  for (long long b0 = 0; ok && b0 < n; b0 += block * nt) {
    std::vector<std::string> out(nt);
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) {
      const long long r0 = b0 + t * block, r1 = std::min(n, r0 + block);
      if (r0 >= r1) break;
      th.emplace_back([&, t, r0, r1] {
        std::string& s = out[t];
        s.reserve(static_cast<size_t>(r1 - r0) * 256);
        for (long long r = r0; r < r1; ++r) fmt(r, s);
      });
    }
    for (auto& x : th) x.join();
    for (int t = 0; t < nt && ok; ++t) ok = std::fwrite(out[t].data(), 1, out[t].size(), f) == out[t].size();
  }
  ok = std::fclose(f) == 0 && ok;
  return ok;
}

int kind_of(const ecg_run_config& c)
{
  switch (c.problem) {
    case ECG_PROBLEM_GRESHO_VORTEX:
      return ecg_out::K_GRESHO;
    case ECG_PROBLEM_TORO1:
      return ecg_out::K_TORO;
    case ECG_PROBLEM_RIEMANN_QUADRANT:
      return ecg_out::K_QUADRANT;
    case ECG_PROBLEM_ADVECTION_BLOB:
      return ecg_out::K_BLOB;
    default:
      return -1;
  }
}

bool reference_bubble(const ecg_run_config& c) { return c.problem == ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_2D; }

}  // namespace

// Column buffers of a context: one for synchronous writes, two slots for
// asynchronous snapshots.
struct EcgOutput {
  struct Slot {
    double* d = nullptr;
    double* h = nullptr;  // pinned
    size_t cap = 0;       // doubles
    cudaEvent_t ready = nullptr, copied = nullptr;
    std::thread writer;
  };
  Slot sync, slot[2];
  int next = 0;
  cudaStream_t side = nullptr;
  ecg_out::MetricPart* d_part = nullptr;
  ecg_out::MetricPart* h_part = nullptr;
  std::atomic<int> failures{0};
};

namespace {

bool slot_reserve(ecg_ctx* c, EcgOutput::Slot& s, size_t doubles)
{
  if (s.cap >= doubles) return true;
  cudaFree(s.d);
  cudaFreeHost(s.h);
  s.d = nullptr;
  s.h = nullptr;
  s.cap = 0;
  if (!ecgi::cuda_ok(c, cudaMalloc(&s.d, doubles * sizeof(double)), "output columns")) return false;
  if (!ecgi::cuda_ok(c, cudaMallocHost(&s.h, doubles * sizeof(double)), "output columns (host)")) return false;
  if (!s.ready && !ecgi::cuda_ok(c, cudaEventCreateWithFlags(&s.ready, cudaEventDisableTiming), "event")) return false;
  if (!s.copied && !ecgi::cuda_ok(c, cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming), "event")) return false;
  s.cap = doubles;
  return true;
}

EcgOutput* output_of(ecg_ctx* c)
{
  if (!c->out) {
    c->out = new EcgOutput();
    if (cudaStreamCreateWithFlags(&c->out->side, cudaStreamNonBlocking) != cudaSuccess) c->out->side = nullptr;
  }
  return c->out;
}

// Columns of the current state into s.d on the context's stream.
bool launch_fields(ecg_ctx* c, EcgOutput::Slot& s, int kind, double time)
{
  const long long n = static_cast<long long>(c->grid.nx) * c->grid.ny;
  if (!slot_reserve(c, s, static_cast<size_t>(kCols) * n)) return false;
  const EcgFvParams P = ecgi::fv_params(c, false);
  const EcgProblem pr = ecgi::problem_of(c, false);
  long long blocks = (n + ecg_out::kNT - 1) / ecg_out::kNT;
  if (blocks > 148LL * 16) blocks = 148LL * 16;
  ecg_out::fields_kernel<<<static_cast<int>(blocks), ecg_out::kNT, 0, c->stream>>>(P, pr, c->cur_state(), kind, time,
                                                                                     s.d);
  return ecgi::cuda_ok(c, cudaGetLastError(), "output columns");
}

bool fetch_sync(ecg_ctx* c, EcgOutput::Slot& s)
{
  const long long n = static_cast<long long>(c->grid.nx) * c->grid.ny;
  if (!ecgi::cuda_ok(c, cudaMemcpyAsync(s.h, s.d, sizeof(double) * kCols * n, cudaMemcpyDeviceToHost, c->stream),
                     "output columns copy"))
    return false;
  return ecgi::cuda_ok(c, cudaStreamSynchronize(c->stream), "output columns copy");
}

std::string snapshot_name(const std::string& dir, int index, double time, int step)
{
  // shock_density_bubble_snapshot_filename (io/output_cases.hpp:405-420)
  char t[64];
  std::snprintf(t, sizeof(t), "%.6f", time);
  std::string tl = t;
  std::replace(tl.begin(), tl.end(), '.', 'p');
  char b[96];
  std::snprintf(b, sizeof(b), "/snapshot_%02d_t%s_step%06d.csv", index, tl.c_str(), step);
  return dir + b;
}

// write_shock_density_bubble_snapshot (io/output_cases.hpp:422-487) from host columns.
bool write_snapshot_file(const ecg_run_config cfg, const EcgGrid g, const double* h, const std::string& dir, int index,
                         int step, double time)
{
  std::error_code ec;
  std::filesystem::create_directories(dir, ec);
  if (ec) return false;
  const long long n = static_cast<long long>(g.nx) * g.ny;
  const std::string scheme = bubble_scheme_name(cfg);
  const char* rlabel = cfg.method == ECG_METHOD_IMEX ? "imex_pressure_split" : riemann_label(cfg.riemann);
  const std::string header =
      "source_case_id,step,time,i,j,x,y,rho,u,v,pressure,internal_energy,"
      "schlieren,density_bubble_indicator,density_bubble_area_threshold,gamma,"
      "method,scheme_name,riemann,spatial_order,validation_claim,gfm_used,"
      "level_set_used,material_count,cylindrical_source_used,"
      "geometric_source_form\n";
  return write_rows(snapshot_name(dir, index, time, step), header, n, [&](long long r, std::string& s) {
    const int j = static_cast<int>(r / g.nx), i = static_cast<int>(r - static_cast<long long>(j) * g.nx);
    const double x = g.plo_x + (static_cast<double>(i) + 0.5) * g.dx;
    const double y = g.plo_y + (static_cast<double>(j) + 0.5) * g.dy;
    const double rho = h[r];
    Row w{s};
    w.t(kBubbleCaseId).c().i(step).c().d(time).c().i(i).c().i(j).c().d(x).c().d(y).c().d(rho).c().d(h[n + r]).c();
    w.d(h[2 * n + r]).c().d(h[3 * n + r]).c().d(h[4 * n + r]).c().d(h[5 * n + r]).c().i(rho < ecg_out::kBubbleThreshold ? 1 : 0).c();
    w.d(ecg_out::kBubbleThreshold).c().d(cfg.gamma).c().t(method_label(cfg.method)).c().t(scheme.c_str()).c();
    w.t(rlabel).c().i(cfg.spatial_order).c().t(kBubbleClaim).t(",false,false,1,false,none\n");
  });
}

}  // namespace

void output_destroy(EcgOutput* o)
{
  if (!o) return;
  for (auto& s : o->slot)
    if (s.writer.joinable()) s.writer.join();
  for (EcgOutput::Slot* s : {&o->sync, &o->slot[0], &o->slot[1]}) {
    cudaFree(s->d);
    cudaFreeHost(s->h);
    if (s->ready) cudaEventDestroy(s->ready);
    if (s->copied) cudaEventDestroy(s->copied);
  }
  cudaFree(o->d_part);
  cudaFreeHost(o->h_part);
  if (o->side) cudaStreamDestroy(o->side);
  delete o;
}

extern "C" {

ecg_status ecg_write_final_csv(ecg_ctx* c, const char* path, const ecg_output_info* info)
{
  if (!c || !path || !info) return ECG_ERR_BAD_ARG;
  if (!c->uploaded) return ECG_ERR_NOT_READY;
  const ecg_run_config& cfg = c->cfg;
  const int kind = kind_of(cfg);
  if (kind < 0) {
    c->err = "no final CSV for this problem (io/output_cases.hpp writes Gresho, Toro, quadrant and blob files)";
    return ECG_ERR_UNSUPPORTED;
  }
  cudaSetDevice(c->device);
  EcgOutput* o = output_of(c);
  if (!launch_fields(c, o->sync, kind, info->time) || !fetch_sync(c, o->sync)) return ECG_ERR_CUDA;
  const EcgGrid g = c->grid;
  const long long n = static_cast<long long>(g.nx) * g.ny;
  const double* h = o->sync.h;
  const bool imex = cfg.method == ECG_METHOD_IMEX;
  const int step = info->step;
  const double time = info->time;
  auto xy = [&](long long r, int& i, int& j, double& x, double& y) {
    j = static_cast<int>(r / g.nx);
    i = static_cast<int>(r - static_cast<long long>(j) * g.nx);
    x = g.plo_x + (static_cast<double>(i) + 0.5) * g.dx;
    y = g.plo_y + (static_cast<double>(j) + 0.5) * g.dy;
  };
  bool ok = false;
  if (kind == ecg_out::K_GRESHO) {
    // write_gresho_final_csv (io/output_cases.hpp:16-73)
    const std::string header =
        "x,y,rho,u,v,pressure,exact_rho,exact_u,exact_v,exact_pressure,"
        "density_error,velocity_error,pressure_error,pressure_perturbation_error,"
        "time,step,mach,method,riemann,imex_form,imex_predictor_flux,imex_predictor_dissipation,"
        "spatial_order,slope_limiter,"
        "imex_trial_density_run_min,"
        "imex_high_trial_pressure_run_min,imex_high_trial_internal_energy_run_min\n";
    const double p0 = cfg.pressure;
    ok = write_rows(path, header, n, [&](long long r, std::string& s) {
      int i, j;
      double x, y;
      xy(r, i, j, x, y);
      const double rho = h[r], u = h[n + r], v = h[2 * n + r], p = h[3 * n + r];
      const double er = h[4 * n + r], eu = h[5 * n + r], ev = h[6 * n + r], ep = h[7 * n + r];
      const double du = u - eu, dv = v - ev;
      Row w{s};
      w.d(x).c().d(y).c().d(rho).c().d(u).c().d(v).c().d(p).c().d(er).c().d(eu).c().d(ev).c().d(ep).c();
      w.d(rho - er).c().d(std::sqrt(du * du + dv * dv)).c().d(p - ep).c().d((p - p0) - (ep - p0)).c();
      w.d(time).c().i(step).c().d(cfg.mach).c().t(method_label(cfg.method)).c();
      w.t(imex ? "not_applicable" : riemann_label(cfg.riemann)).c().t(imex ? kImexForm : "not_applicable").c();
      w.t(imex ? kImexPredictorFlux : "not_applicable").c().t(imex ? kImexPredictorDissipation : "not_applicable").c();
      w.i(cfg.spatial_order).c().t(limiter_label(cfg.slope_limiter)).c();
      w.d(info->trial_density_min).c().d(info->trial_pressure_min).c().d(info->trial_internal_energy_min).t("\n");
    });
  } else if (kind == ecg_out::K_TORO) {
    // write_toro_final_csv (io/output_cases.hpp:75-111): exact columns are NaN there
    const std::string header =
        "i,j,x,y,rho,u,v,p,exact_rho,exact_u,exact_v,exact_p,"
        "rho_error,u_error,v_error,p_error\n";
    ok = write_rows(path, header, n, [&](long long r, std::string& s) {
      int i, j;
      double x, y;
      xy(r, i, j, x, y);
      Row w{s};
      w.i(i).c().i(j).c().d(x).c().d(y).c().d(h[r]).c().d(h[n + r]).c().d(h[2 * n + r]).c().d(h[3 * n + r]);
      w.t(",nan,nan,nan,nan,nan,nan,nan,nan\n");
    });
  } else if (kind == ecg_out::K_QUADRANT) {
    // write_riemann_quadrant_final_csv (io/output_cases.hpp:113-157)
    const std::string header =
        "i,j,x,y,rho,u,v,p,initial_rho,initial_u,initial_v,initial_p,"
        "time,step,method,riemann,spatial_order,slope_limiter,"
        "field_boundary,geometry_is_periodic_x,geometry_is_periodic_y,"
        "quadrant_case,claim_limit\n";
    const char* fb = cfg.field_boundary == ECG_FIELD_BOUNDARY_EXACT_DIRICHLET ? "exact_dirichlet" : "outflow";
    ok = write_rows(path, header, n, [&](long long r, std::string& s) {
      int i, j;
      double x, y;
      xy(r, i, j, x, y);
      Row w{s};
      w.i(i).c().i(j).c().d(x).c().d(y).c();
      for (int k = 0; k < 8; ++k) w.d(h[k * n + r]).c();
      w.d(time).c().i(step).c().t(method_label(cfg.method)).c();
      w.t(imex ? "imex_pressure_split" : riemann_label(cfg.riemann)).c().i(cfg.spatial_order).c();
      w.t(limiter_label(cfg.slope_limiter)).c().t(fb).c().i(cfg.is_periodic[0] != 0).c().i(cfg.is_periodic[1] != 0).c();
      w.t("liska_wendroff_clawpack_quadrant,genuine_2d_visual_finite_smoke_no_exact_solution\n");
    });
  } else {
    // write_advection_blob_final_csv (io/output_cases.hpp:159-208)
    const std::string header =
        "x,y,rho,u,v,pressure,exact_rho,exact_u,exact_v,exact_pressure,"
        "density_error,velocity_error,pressure_error,time,step,method,riemann,"
        "spatial_order,slope_limiter,geometry_is_periodic_x,geometry_is_periodic_y\n";
    ok = write_rows(path, header, n, [&](long long r, std::string& s) {
      int i, j;
      double x, y;
      xy(r, i, j, x, y);
      const double rho = h[r], u = h[n + r], v = h[2 * n + r], p = h[3 * n + r];
      const double er = h[4 * n + r], eu = h[5 * n + r], ev = h[6 * n + r], ep = h[7 * n + r];
      const double du = u - eu, dv = v - ev;
      Row w{s};
      w.d(x).c().d(y).c().d(rho).c().d(u).c().d(v).c().d(p).c().d(er).c().d(eu).c().d(ev).c().d(ep).c();
      w.d(rho - er).c().d(std::sqrt(du * du + dv * dv)).c().d(p - ep).c().d(time).c().i(step).c();
      w.t(method_label(cfg.method)).c().t(imex ? "imex_pressure_split" : riemann_label(cfg.riemann)).c();
      w.i(cfg.spatial_order).c().t(limiter_label(cfg.slope_limiter)).c().i(cfg.is_periodic[0] != 0).c();
      w.i(cfg.is_periodic[1] != 0).t("\n");
    });
  }
  if (!ok) {
    c->err = std::string("cannot write ") + path;
    return ECG_ERR_IO;
  }
  return ECG_OK;
}

ecg_status ecg_shock_bubble_metrics(ecg_ctx* c, double time, ecg_bubble_metrics* out)
{
  (void)time;  // the bubble's ghost states do not depend on time
  if (!c || !out) return ECG_ERR_BAD_ARG;
  if (!c->uploaded) return ECG_ERR_NOT_READY;
  if (c->cfg.problem != ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_2D && c->cfg.problem != ECG_PROBLEM_SHOCK_BUBBLE_MACH122) {
    c->err = "bubble metrics need a shock-density-bubble problem";
    return ECG_ERR_UNSUPPORTED;
  }
  cudaSetDevice(c->device);
  EcgOutput* o = output_of(c);
  const int nb = ecg_out::kMetricBlocks;
  if (!o->d_part) {
    if (!ecgi::cuda_ok(c, cudaMalloc(&o->d_part, sizeof(ecg_out::MetricPart) * nb), "metrics")) return ECG_ERR_CUDA;
    if (!ecgi::cuda_ok(c, cudaMallocHost(&o->h_part, sizeof(ecg_out::MetricPart) * nb), "metrics")) return ECG_ERR_CUDA;
  }
  const EcgFvParams P = ecgi::fv_params(c, false);
  ecg_out::metrics_kernel<<<nb, ecg_out::kNT, 0, c->stream>>>(P, c->cur_state(), o->d_part);
  if (!ecgi::cuda_ok(c, cudaGetLastError(), "metrics") ||
      !ecgi::cuda_ok(c, cudaMemcpyAsync(o->h_part, o->d_part, sizeof(ecg_out::MetricPart) * nb, cudaMemcpyDeviceToHost,
                                        c->stream),
                     "metrics") ||
      !ecgi::cuda_ok(c, cudaStreamSynchronize(c->stream), "metrics"))
    return ECG_ERR_CUDA;
  const double inf = std::numeric_limits<double>::infinity();
  ecg_out::MetricPart m{inf, -inf, inf, -inf, inf, 0.0, 0.0, 0.0, 0.0, 0};
  for (int b = 0; b < nb; ++b) {
    const auto& p = o->h_part[b];
    m.rho_min = std::min(m.rho_min, p.rho_min);
    m.rho_max = std::max(m.rho_max, p.rho_max);
    m.p_min = std::min(m.p_min, p.p_min);
    m.p_max = std::max(m.p_max, p.p_max);
    m.ie_min = std::min(m.ie_min, p.ie_min);
    m.area += p.area;
    m.cx_sum += p.cx_sum;
    m.cy_sum += p.cy_sum;
    m.schlieren = std::max(m.schlieren, p.schlieren);
    m.nonfinite += p.nonfinite;
  }
  std::memset(out, 0, sizeof(*out));
  out->rho_min = m.rho_min;
  out->rho_max = m.rho_max;
  out->pressure_min = m.p_min;
  out->pressure_max = m.p_max;
  out->internal_energy_min = m.ie_min;
  out->density_bubble_area = m.area;
  out->density_bubble_area_threshold = ecg_out::kBubbleThreshold;
  const double nan = std::numeric_limits<double>::quiet_NaN();
  out->density_bubble_centroid_x = m.area > 0.0 ? m.cx_sum / m.area : nan;
  out->density_bubble_centroid_y = m.area > 0.0 ? m.cy_sum / m.area : nan;
  out->schlieren_max = m.schlieren;
  out->nonfinite_count = static_cast<int32_t>(m.nonfinite);
  return ECG_OK;
}

ecg_status ecg_write_bubble_snapshot(ecg_ctx* c, const char* dir, int32_t index, int32_t step, double time,
                                     int32_t async)
{
  if (!c || !dir) return ECG_ERR_BAD_ARG;
  if (!c->uploaded) return ECG_ERR_NOT_READY;
  if (!reference_bubble(c->cfg)) {
    c->err = "bubble snapshots are written for shock_density_bubble_2d";
    return ECG_ERR_UNSUPPORTED;
  }
  cudaSetDevice(c->device);
  EcgOutput* o = output_of(c);
  if (!async || !o->side) {
    if (!launch_fields(c, o->sync, ecg_out::K_BUBBLE, time) || !fetch_sync(c, o->sync)) return ECG_ERR_CUDA;
    if (!write_snapshot_file(c->cfg, c->grid, o->sync.h, dir, index, step, time)) {
      c->err = std::string("cannot write a snapshot into ") + dir;
      return ECG_ERR_IO;
    }
    return ECG_OK;
  }
  EcgOutput::Slot& s = o->slot[o->next];
  if (s.writer.joinable()) s.writer.join();  // both slots busy: wait for the older file
  if (!launch_fields(c, s, ecg_out::K_BUBBLE, time)) return ECG_ERR_CUDA;
  const long long n = static_cast<long long>(c->grid.nx) * c->grid.ny;
  if (!ecgi::cuda_ok(c, cudaEventRecord(s.ready, c->stream), "snapshot") ||
      !ecgi::cuda_ok(c, cudaStreamWaitEvent(o->side, s.ready, 0), "snapshot") ||
      !ecgi::cuda_ok(c, cudaMemcpyAsync(s.h, s.d, sizeof(double) * kCols * n, cudaMemcpyDeviceToHost, o->side),
                     "snapshot copy") ||
      !ecgi::cuda_ok(c, cudaEventRecord(s.copied, o->side), "snapshot"))
    return ECG_ERR_CUDA;
  const ecg_run_config cfg = c->cfg;
  const EcgGrid g = c->grid;
  const std::string d = dir;
  const int dev = c->device;
  s.writer = std::thread([o, &s, cfg, g, d, index, step, time, dev] {
    cudaSetDevice(dev);
    const bool ok = cudaEventSynchronize(s.copied) == cudaSuccess &&
                    write_snapshot_file(cfg, g, s.h, d, index, step, time);
    if (!ok) o->failures.fetch_add(1);
  });
  o->next ^= 1;
  return ECG_OK;
}

ecg_status ecg_output_wait(ecg_ctx* c, int32_t* failed)
{
  if (!c) return ECG_ERR_BAD_ARG;
  int f = 0;
  if (c->out) {
    for (auto& s : c->out->slot)
      if (s.writer.joinable()) s.writer.join();
    f = c->out->failures.exchange(0);
  }
  if (failed) *failed = f;
  if (f > 0) {
    c->err = "an asynchronous snapshot could not be written";
    return ECG_ERR_IO;
  }
  return ECG_OK;
}

ecg_status ecg_write_bubble_summary_csv(ecg_ctx* c, const char* path, const ecg_bubble_run* run)
{
  if (!c || !path || !run) return ECG_ERR_BAD_ARG;
  if (!reference_bubble(c->cfg)) {
    c->err = "the bubble summary is written for shock_density_bubble_2d";
    return ECG_ERR_UNSUPPORTED;
  }
  ecg_bubble_metrics m;
  const ecg_status st = ecg_shock_bubble_metrics(c, run->time, &m);
  if (st != ECG_OK) return st;
  const ecg_run_config& cfg = c->cfg;
  // write_shock_density_bubble_summary_csv (io/output_cases.hpp:489-588)
  std::string s =
      "source_case_id,run_id,backend,scheme_family,scheme_name,order,riemann,"
      "gamma,grid_nx,grid_ny,x_lower,x_upper,y_lower,y_upper,shock_initial_x,"
      "post_shock_density,post_shock_velocity,post_shock_pressure,bubble_density,"
      "bubble_center_x,bubble_center_y,bubble_radius,boundary_left,boundary_right,"
      "boundary_bottom,boundary_top,final_time,snapshot_times,status,"
      "failure_category,steps_accepted,steps_rejected,wall_time_sec,dt_min,dt_max,"
      "dt_mean,rho_min,rho_max,pressure_min,pressure_max,internal_energy_min,"
      "nonfinite_count,density_bubble_centroid_x,density_bubble_centroid_y,"
      "density_bubble_area_threshold,schlieren_max,snapshot_status,snapshot_dir,"
      "validation_claim,gfm_used,level_set_used,material_count,"
      "cylindrical_source_used,geometric_source_form\n";
  const std::string scheme = bubble_scheme_name(cfg);
  const std::string run_id = scheme + "_" + std::to_string(cfg.n_cell[0]) + "x" + std::to_string(cfg.n_cell[1]);
  const auto str = [](const char* v) { return std::string(v ? v : ""); };
  Row w{s};
  w.t(kBubbleCaseId).c().t(csv_escape(run_id).c_str()).t(",amrex_single_level,").t(method_label(cfg.method)).c();
  w.t(csv_escape(scheme).c_str()).c().t(csv_escape(cfg.method == ECG_METHOD_IMEX ? "T1/S2" : "O" + std::to_string(cfg.spatial_order)).c_str()).c();
  w.t(cfg.method == ECG_METHOD_IMEX ? "imex_pressure_split" : riemann_label(cfg.riemann)).c().d(cfg.gamma).c();
  w.i(cfg.n_cell[0]).c().i(cfg.n_cell[1]).c().d(cfg.prob_lo[0]).c().d(cfg.prob_hi[0]).c().d(cfg.prob_lo[1]).c();
  w.d(cfg.prob_hi[1]).c().d(kBubbleShockX).c().d(kPostShock[0]).c().d(kPostShock[1]).c().d(kPostShock[3]).c();
  w.d(kBubbleRho).c().d(kBubbleCx).c().d(kBubbleCy).c().d(kBubbleR);
  w.t(",fixed_post_shock_inflow,outflow_zero_gradient,reflective_symmetry,outflow_zero_gradient,");
  w.d(cfg.stop_time).c().t(csv_escape(str(run->snapshot_times)).c_str()).c().t(str(run->status).c_str()).c();
  w.t(str(run->failure_category).c_str()).c().i(run->steps_accepted).c().i(run->steps_rejected).c();
  w.d(run->wall_time_sec).c().d(run->dt_min).c().d(run->dt_max).c().d(run->dt_mean).c().d(m.rho_min).c();
  w.d(m.rho_max).c().d(m.pressure_min).c().d(m.pressure_max).c().d(m.internal_energy_min).c().i(m.nonfinite_count).c();
  w.d(m.density_bubble_centroid_x).c().d(m.density_bubble_centroid_y).c().d(m.density_bubble_area_threshold).c();
  w.d(m.schlieren_max).c().t(str(run->snapshot_status).c_str()).c().t(csv_escape(str(run->snapshot_dir)).c_str()).c();
  w.t(kBubbleClaim).t(",false,false,1,false,none\n");
  std::FILE* f = std::fopen(path, "wb");
  const bool ok = f && std::fwrite(s.data(), 1, s.size(), f) == s.size();
  if (f && std::fclose(f) != 0) return ECG_ERR_IO;
  if (!ok) {
    c->err = std::string("cannot write ") + path;
    return ECG_ERR_IO;
  }
  return ECG_OK;
}

}  // extern "C"
