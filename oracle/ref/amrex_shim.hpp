// Minimal single-box stand-in for the parts of AMReX that the euler_compare
// hot-path headers use.  TEST INFRASTRUCTURE ONLY: it lets the reference's own
// numerics headers (amrex/apps/euler_compare/src/euler_compare/**) compile with
// plain g++ into oracle/_ref/, so the CPU oracle is the reference's code itself.
//
// Semantics follow AMReX where the numerics can observe them:
//  * Array4 indexing p[(i-lo.x) + (j-lo.y)*jstride + n*nstride]
//    (external/AMReX/Src/Base/AMReX_Array4.H).
//  * Geometry cell size dx = (prob_hi - prob_lo) / n  (AMReX_Geometry.cpp:527).
//  * ReduceOpSum/Min/Max init 0 / numeric_limits::max() / lowest() and
//    local_update d+=s, d=min(d,s), d=max(d,s)  (AMReX_Reduce.H:283-380);
//    CPU eval visits cells k, j, i with i fastest (AMReX_Reduce.H:1380-1395).
//  * amrex::min/max are std::min/std::max (AMReX_Algorithm.H:20-56).
//  * FillBoundary(periodicity) fills a ghost cell iff its periodic image lies
//    in the valid domain (single box covering the domain).
// Everything is one box: the reference's numerics do not depend on the box
// decomposition except through the order of floating-point sums.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include <thread>

#define AMREX_SPACEDIM 2
#define AMREX_GPU_HOST_DEVICE
#define AMREX_GPU_DEVICE
#define AMREX_FORCE_INLINE inline
#define AMREX_D_DECL(a, b, c) a, b
#define BL_PROFILE(x)

namespace amrex {

using Real = double;
using Long = long long;
template <class T>
using Vector = std::vector<T>;
template <class T, std::size_t N>
using Array = std::array<T, N>;

template <class T, int N>
struct GpuArray {
  T arr[N];
  const T& operator[](int i) const noexcept { return arr[i]; }
  T& operator[](int i) noexcept { return arr[i]; }
};

template <class T>
inline const T& min(const T& a, const T& b) noexcept { return std::min(a, b); }
template <class T, class... Ts>
inline const T& min(const T& a, const T& b, const Ts&... c) noexcept { return min(min(a, b), c...); }
template <class T>
inline const T& max(const T& a, const T& b) noexcept { return std::max(a, b); }
template <class T, class... Ts>
inline const T& max(const T& a, const T& b, const Ts&... c) noexcept { return max(max(a, b), c...); }

[[noreturn]] inline void Abort(const std::string& msg) { throw std::runtime_error(msg); }

// Print: output is discarded unless a caller collects it (print_sink()),
// with doubles written as %.17g (the precision the reference's driver
// reports at) and stream manipulators ignored.  iostreams are kept out of
// every path the oracle calls.
inline std::string*& print_sink()
{
  static std::string* sink = nullptr;
  return sink;
}
// A driver executable (Initialize) prints to stdout instead.
inline bool& print_to_stdout()
{
  static bool on = false;
  return on;
}
inline void print_text(const char* s, std::size_t n)
{
  if (print_to_stdout()) std::fwrite(s, 1, n, stdout);
  else if (print_sink()) print_sink()->append(s, n);
}
struct Print {
  template <class T>
  Print& operator<<(const T&) { return *this; }
  Print& operator<<(const char* s)
  {
    print_text(s, std::strlen(s));
    return *this;
  }
  Print& operator<<(const std::string& s)
  {
    print_text(s.data(), s.size());
    return *this;
  }
  Print& operator<<(char c)
  {
    print_text(&c, 1);
    return *this;
  }
  Print& operator<<(double v) { return num("%.17g", v); }
  Print& operator<<(float v) { return num("%.17g", static_cast<double>(v)); }
  Print& operator<<(int v) { return inum(v); }
  Print& operator<<(long v) { return inum(v); }
  Print& operator<<(long long v) { return inum(v); }
  Print& operator<<(unsigned v) { return inum(static_cast<long long>(v)); }
  Print& operator<<(bool v) { return inum(v ? 1 : 0); }

 private:
  Print& num(const char* fmt, double v)
  {
    char b[64];
    const int n = std::snprintf(b, sizeof(b), fmt, v);
    print_text(b, static_cast<std::size_t>(n));
    return *this;
  }
  Print& inum(long long v)
  {
    char b[32];
    const int n = std::snprintf(b, sizeof(b), "%lld", v);
    print_text(b, static_cast<std::size_t>(n));
    return *this;
  }
};

struct Dim3 { int x, y, z; };

struct IntVect {
  int v[2] = {0, 0};
  IntVect() = default;
  IntVect(int a, int b) { v[0] = a; v[1] = b; }
  int operator[](int d) const noexcept { return v[d]; }
  int& operator[](int d) noexcept { return v[d]; }
};

struct Box {
  IntVect lo, hi;
  Box() = default;
  Box(const IntVect& l, const IntVect& h) : lo(l), hi(h) {}
  const IntVect& smallEnd() const noexcept { return lo; }
  const IntVect& bigEnd() const noexcept { return hi; }
  int smallEnd(int d) const noexcept { return lo[d]; }
  int bigEnd(int d) const noexcept { return hi[d]; }
  int length(int d) const noexcept { return hi[d] - lo[d] + 1; }
  Box grow(const IntVect& g) const { return Box(IntVect(lo[0] - g[0], lo[1] - g[1]), IntVect(hi[0] + g[0], hi[1] + g[1])); }
  bool contains(int i, int j) const noexcept { return i >= lo[0] && i <= hi[0] && j >= lo[1] && j <= hi[1]; }
};
inline Dim3 lbound(const Box& b) noexcept { return Dim3{b.lo[0], b.lo[1], 0}; }
inline Dim3 ubound(const Box& b) noexcept { return Dim3{b.hi[0], b.hi[1], 0}; }

template <class T>
struct Array4 {
  T* p = nullptr;
  Long jstride = 0;
  Long nstride = 0;
  Dim3 begin{0, 0, 0};
  int ncomp = 0;
  Array4() = default;
  Array4(T* p_, Long js, Long ns, Dim3 b, int nc) : p(p_), jstride(js), nstride(ns), begin(b), ncomp(nc) {}
  template <class U, class = std::enable_if_t<std::is_same<std::add_const_t<U>, T>::value && !std::is_same<U, T>::value>>
  Array4(const Array4<U>& o) : p(o.p), jstride(o.jstride), nstride(o.nstride), begin(o.begin), ncomp(o.ncomp) {}
  T& operator()(int i, int j, int) const noexcept { return p[(i - begin.x) + (j - begin.y) * jstride]; }
  T& operator()(int i, int j, int, int n) const noexcept {
    return p[(i - begin.x) + (j - begin.y) * jstride + n * nstride];
  }
};

struct RealBox {
  Real xlo[2], xhi[2];
  RealBox(const Real* lo, const Real* hi) { for (int d = 0; d < 2; ++d) { xlo[d] = lo[d]; xhi[d] = hi[d]; } }
  Real length(int d) const noexcept { return xhi[d] - xlo[d]; }
};

struct CoordSys { enum CoordType { cartesian = 0 }; };

struct Periodicity { int period[2] = {0, 0}; };

struct Geometry {
  Box domain;
  Real plo[2] = {0, 0}, phi[2] = {1, 1}, dx[2] = {1, 1};
  int per[2] = {0, 0};
  Geometry() = default;
  Geometry(const Box& dom, const RealBox* rb, int, const int* is_per) : domain(dom) {
    for (int k = 0; k < 2; ++k) {
      plo[k] = rb->xlo[k];
      phi[k] = rb->xhi[k];
      dx[k] = rb->length(k) / (Real(domain.length(k)));
      per[k] = is_per[k];
    }
  }
  GpuArray<Real, 2> CellSizeArray() const noexcept { return GpuArray<Real, 2>{{dx[0], dx[1]}}; }
  GpuArray<Real, 2> ProbLoArray() const noexcept { return GpuArray<Real, 2>{{plo[0], plo[1]}}; }
  GpuArray<Real, 2> ProbHiArray() const noexcept { return GpuArray<Real, 2>{{phi[0], phi[1]}}; }
  const Box& Domain() const noexcept { return domain; }
  bool isPeriodic(int d) const noexcept { return per[d] != 0; }
  Periodicity periodicity() const noexcept {
    Periodicity pr;
    for (int d = 0; d < 2; ++d) { pr.period[d] = per[d] ? domain.length(d) : 0; }
    return pr;
  }
};

struct BoxArray {
  Box box;
  BoxArray() = default;
  explicit BoxArray(const Box& b) : box(b) {}
  void maxSize(int) {}
};
struct DistributionMapping {
  DistributionMapping() = default;
  explicit DistributionMapping(const BoxArray&) {}
};

class MFIter;

class MultiFab {
 public:
  BoxArray ba;
  Box valid, grown;
  int ncomp = 0, ng = 0;
  Long jstride = 0, nstride = 0;
  std::vector<Real> data;

  MultiFab() = default;
  MultiFab(const BoxArray& ba_, const DistributionMapping&, int nc, int ngrow)
      : ba(ba_), valid(ba_.box), ncomp(nc), ng(ngrow) {
    grown = valid.grow(IntVect(ng, ng));
    jstride = grown.length(0);
    nstride = jstride * grown.length(1);
    data.assign(static_cast<std::size_t>(nstride * ncomp), 0.0);
  }
  Array4<Real> array(const MFIter&) { return Array4<Real>(data.data(), jstride, nstride, lbound(grown), ncomp); }
  Array4<const Real> array(const MFIter&) const { return const_array_impl(); }
  Array4<const Real> const_array(const MFIter&) const { return const_array_impl(); }
  Array4<Real> arr() { return Array4<Real>(data.data(), jstride, nstride, lbound(grown), ncomp); }
  Array4<const Real> const_array_impl() const {
    return Array4<const Real>(data.data(), jstride, nstride, lbound(grown), ncomp);
  }
  IntVect nGrowVect() const noexcept { return IntVect(ng, ng); }
  int nComp() const noexcept { return ncomp; }
  const BoxArray& boxArray() const noexcept { return ba; }
  DistributionMapping DistributionMap() const { return DistributionMapping(ba); }

  void FillBoundary(const Periodicity& per) {
    auto a = arr();
    const int nx = valid.length(0), ny = valid.length(1);
    for (int n = 0; n < ncomp; ++n) {
      for (int j = grown.lo[1]; j <= grown.hi[1]; ++j) {
        for (int i = grown.lo[0]; i <= grown.hi[0]; ++i) {
          if (valid.contains(i, j)) { continue; }
          int ii = i, jj = j;
          if (per.period[0] != 0) { ii = ((i - valid.lo[0]) % nx + nx) % nx + valid.lo[0]; }
          if (per.period[1] != 0) { jj = ((j - valid.lo[1]) % ny + ny) % ny + valid.lo[1]; }
          if (valid.contains(ii, jj)) { a(i, j, 0, n) = a(ii, jj, 0, n); }
        }
      }
    }
  }
  Real sum(int comp) const {
    auto a = const_array_impl();
    Real s = 0.0;
    for (int j = valid.lo[1]; j <= valid.hi[1]; ++j) {
      for (int i = valid.lo[0]; i <= valid.hi[0]; ++i) { s += a(i, j, 0, comp); }
    }
    return s;
  }
  static void Copy(MultiFab& dst, const MultiFab& src, int scomp, int dcomp, int nc, int ngrow) {
    auto d = dst.arr();
    auto s = src.const_array_impl();
    const Box b = dst.valid.grow(IntVect(ngrow, ngrow));
    for (int n = 0; n < nc; ++n) {
      for (int j = b.lo[1]; j <= b.hi[1]; ++j) {
        for (int i = b.lo[0]; i <= b.hi[0]; ++i) { d(i, j, 0, dcomp + n) = s(i, j, 0, scomp + n); }
      }
    }
  }
};

class MFIter {
 public:
  const MultiFab* mf;
  bool valid_ = true;
  explicit MFIter(const MultiFab& m, bool = false) : mf(&m) {}
  bool isValid() const noexcept { return valid_; }
  void operator++() { valid_ = false; }
  Box validbox() const { return mf->valid; }
  Box growntilebox(const IntVect& g) const { return mf->valid.grow(g); }
  int LocalIndex() const { return 0; }
};

// Row-parallel execution for the timed CPU baseline: ECG_REF_THREADS host
// threads share the rows of a box (default 1 = AMReX's serial CPU order).
// Every cell is written by exactly one iteration, so results do not depend on
// the thread count.
inline int shim_threads() {
  const char* e = std::getenv("ECG_REF_THREADS");
  const int v = e ? std::atoi(e) : 1;
  return v < 1 ? 1 : v;
}
template <class Body>
inline void parallel_rows(int lo, int hi, Body&& body) {
  const int nt = shim_threads();
  const int n = hi - lo + 1;
  if (nt <= 1 || n < 2 * nt) {
    for (int j = lo; j <= hi; ++j) body(0, j);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(static_cast<std::size_t>(nt));
  for (int t = 0; t < nt; ++t) {
    const int a = lo + static_cast<int>(static_cast<long long>(t) * n / nt);
    const int b = lo + static_cast<int>(static_cast<long long>(t + 1) * n / nt);
    th.emplace_back([&body, a, b, t] { for (int j = a; j < b; ++j) body(t, j); });
  }
  for (auto& x : th) x.join();
}

template <class F>
inline void ParallelFor(const Box& b, F&& f) {
  parallel_rows(b.lo[1], b.hi[1], [&](int, int j) {
    for (int i = b.lo[0]; i <= b.hi[0]; ++i) { f(i, j, 0); }
  });
}
template <class F>
inline void ParallelFor(const Box& b, int ncomp, F&& f) {
  for (int n = 0; n < ncomp; ++n) {
    parallel_rows(b.lo[1], b.hi[1], [&](int, int j) {
      for (int i = b.lo[0]; i <= b.hi[0]; ++i) { f(i, j, 0, n); }
    });
  }
}

struct ReduceOpSum {
  template <class T> void local_update(T& d, const T& s) const noexcept { d += s; }
  template <class T> void init(T& t) const noexcept { t = 0; }
};
struct ReduceOpMin {
  template <class T> void local_update(T& d, const T& s) const noexcept { d = amrex::min(d, s); }
  template <class T> void init(T& t) const noexcept { t = std::numeric_limits<T>::max(); }
};
struct ReduceOpMax {
  template <class T> void local_update(T& d, const T& s) const noexcept { d = amrex::max(d, s); }
  template <class T> void init(T& t) const noexcept { t = std::numeric_limits<T>::lowest(); }
};

template <class... Ps>
struct ReduceOps {
  template <class Tuple, std::size_t... I>
  static void init_all(Tuple& t, std::index_sequence<I...>) { (Ps{}.init(std::get<I>(t)), ...); }
  template <class Tuple, std::size_t... I>
  static void update_all(Tuple& d, const Tuple& s, std::index_sequence<I...>) {
    (Ps{}.local_update(std::get<I>(d), std::get<I>(s)), ...);
  }
  // Serial: cells in AMReX's CPU order (i fastest).  Threaded: partials over
  // contiguous row blocks, combined in block order (min, max and integer sums
  // are unchanged; floating-point sums may round differently).
  template <class D, class F>
  void eval(const Box& box, D& data, F&& f) {
    typename D::Type rr;
    init_all(rr, std::index_sequence_for<Ps...>{});
    const int nt = shim_threads();
    std::vector<typename D::Type> part(static_cast<std::size_t>(nt));
    for (auto& p : part) init_all(p, std::index_sequence_for<Ps...>{});
    parallel_rows(box.lo[1], box.hi[1], [&](int t, int j) {
      for (int i = box.lo[0]; i <= box.hi[0]; ++i) {
        const typename D::Type v = f(i, j, 0);
        update_all(part[static_cast<std::size_t>(t)], v, std::index_sequence_for<Ps...>{});
      }
    });
    for (const auto& p : part) update_all(rr, p, std::index_sequence_for<Ps...>{});
    update_all(data.r, rr, std::index_sequence_for<Ps...>{});
  }
};

template <class... Ts>
struct ReduceData {
  using Type = std::tuple<Ts...>;
  Type r;
  template <class... Ps>
  explicit ReduceData(ReduceOps<Ps...>&) { ReduceOps<Ps...>::init_all(r, std::index_sequence_for<Ps...>{}); }
  Type value() const { return r; }
};

template <std::size_t I, class T>
inline decltype(auto) get(T&& t) { return std::get<I>(std::forward<T>(t)); }

// Plotfiles are outside the oracle (the hot path never writes them): the
// writer is a no-op and only the name helper is real.
inline std::string Concatenate(const std::string& root, int num, int mindigits = 5)
{
  char b[32];
  std::snprintf(b, sizeof(b), "%0*d", mindigits, num);
  return root + b;
}
template <class MF, class Names, class Geom>
inline void WriteSingleLevelPlotfile(const std::string&, const MF&, const Names&, const Geom&, Real, int)
{
}

namespace ParallelDescriptor {
inline void ReduceRealSum(Real&) {}
inline void ReduceRealMin(Real&) {}
inline void ReduceRealMax(Real&) {}
inline void ReduceIntSum(int&) {}
inline void ReduceLongSum(Long&) {}
inline int NProcs() { return 1; }
inline bool IOProcessor() { return true; }
}  // namespace ParallelDescriptor

namespace Gpu {
inline void streamSynchronize() {}
}  // namespace Gpu

// ParmParse backed by a process-global key -> values table that the oracle
// fills from "key=value" lines, as AMReX does from argv.
inline std::map<std::string, std::vector<std::string>>& parmparse_table() {
  static std::map<std::string, std::vector<std::string>> t;
  return t;
}
class ParmParse {
 public:
  std::string prefix;
  explicit ParmParse(const std::string& p = "") : prefix(p) {}
  std::string key(const std::string& n) const { return prefix.empty() ? n : prefix + "." + n; }
  const std::vector<std::string>* find(const std::string& n) const {
    auto& t = parmparse_table();
    auto it = t.find(key(n));
    return it == t.end() ? nullptr : &it->second;
  }
  static bool parse_one(const std::string& s, int& out) {
    char* end = nullptr;
    const long v = std::strtol(s.c_str(), &end, 10);
    if (end == s.c_str()) { Abort("ParmParse: cannot parse '" + s + "' as int"); }
    out = static_cast<int>(v);
    return true;
  }
  static bool parse_one(const std::string& s, double& out) {
    char* end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    if (end == s.c_str()) { Abort("ParmParse: cannot parse '" + s + "' as real"); }
    out = v;
    return true;
  }
  static bool parse_one(const std::string& s, std::string& out) { out = s; return true; }
  template <class T>
  bool query(const std::string& n, T& out) const {
    const auto* v = find(n);
    if (v == nullptr || v->empty()) { return false; }
    return parse_one((*v)[0], out);
  }
  int countval(const std::string& n) const {
    const auto* v = find(n);
    return v == nullptr ? 0 : static_cast<int>(v->size());
  }
  template <class T>
  bool queryarr(const std::string& n, std::vector<T>& out, int start, int num) const {
    const auto* v = find(n);
    if (v == nullptr) { return false; }
    for (int k = 0; k < num && start + k < static_cast<int>(v->size()); ++k) {
      parse_one((*v)[start + k], out[k]);
    }
    return true;
  }
};

// The executable's start-up as AMReX does it for the driver: every
// "key=value ..." argument becomes a ParmParse entry (values split at
// whitespace), and Print goes to stdout.
inline void Initialize(int& argc, char**& argv)
{
  auto& table = parmparse_table();
  table.clear();
  for (int a = 1; a < argc; ++a) {
    const std::string arg(argv[a]);
    const auto eq = arg.find('=');
    if (eq == std::string::npos || eq == 0) continue;
    std::vector<std::string> vals;
    std::size_t k = eq + 1;
    while (k < arg.size()) {
      while (k < arg.size() && std::isspace(static_cast<unsigned char>(arg[k]))) ++k;
      std::size_t e = k;
      while (e < arg.size() && !std::isspace(static_cast<unsigned char>(arg[e]))) ++e;
      if (e > k) vals.push_back(arg.substr(k, e - k));
      k = e;
    }
    table[arg.substr(0, eq)] = vals;
  }
  print_to_stdout() = true;
}
inline void Finalize() { std::fflush(stdout); }

}  // namespace amrex
