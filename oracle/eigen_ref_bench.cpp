// eigen_ref_bench.cpp -- times Eigen's own CPU GEMM (the reference implementation of
// the dense product path) on synthetic inputs.  TEST/BENCH INFRASTRUCTURE ONLY: the
// benchmark's CPU-baseline leg and its reference arm run it; the product library
// never does.
//
// It is compiled against the Eigen headers of the reference tree by oracle/Makefile
// (with -fopenmp, so Eigen's parallelize_gemm in
// Eigen/src/Core/products/Parallelizer.h:173-242 splits the product across all
// threads).  The product goes through the public API:
//   C *= beta;  C.noalias() += alpha * op(A) * op(B);
// which reaches generic_product_impl<...,GemmProduct>::scaleAndAddTo
// (Eigen/src/Core/products/GeneralMatrixMatrix.h:476-514) and from there the
// GEBP kernel (Eigen/src/Core/products/GeneralBlockPanelKernel.h:1470-1873).
//
// Modes
//   gemm  : one (possibly transposed, padded-ld) product, repeated --reps times
//   batch : --count independent products with log-uniform sizes in [3,256], 20% of
//           them drawn from the fixed sizes {3,4,6,8}; those use fixed-size
//           Matrix<Scalar,N,N> types, which Eigen evaluates as unrolled
//           coefficient-based products (Eigen/src/Core/GeneralProduct.h:76-80,
//           Eigen/src/Core/ProductEvaluators.h:703-880); the batch loop is an
//           OpenMP parallel for.
// Output: one JSON line with the median seconds per repetition and GFLOP/s.
#include <Eigen/Core>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct Args {
  std::string mode = "gemm";
  char dtype = 'd';
  long m = 512, n = 512, k = 512;
  char ta = 'N', tb = 'N';
  double alpha = 1.0, beta = 0.0;
  long pad = 0;
  int reps = 5;
  int warmup = 1;
  long count = 10000;
  unsigned long long seed = 42;
  double max_seconds = 20.0;
};

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename T>
void fill_uniform(std::vector<T>& v, std::mt19937_64& g) {
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  for (auto& x : v) x = T(u(g));
}

template <typename T>
int run_gemm(const Args& a) {
  using Mat = Eigen::Matrix<T, Eigen::Dynamic, Eigen::Dynamic>;
  using MapM = Eigen::Map<Mat, 0, Eigen::OuterStride<>>;
  const bool tA = (a.ta != 'N' && a.ta != 'n');
  const bool tB = (a.tb != 'N' && a.tb != 'n');
  const long ar = tA ? a.k : a.m, ac = tA ? a.m : a.k;
  const long br = tB ? a.n : a.k, bc = tB ? a.k : a.n;
  const long lda = ar + a.pad, ldb = br + a.pad, ldc = a.m + a.pad;
  std::mt19937_64 g(a.seed);
  std::vector<T> A(size_t(lda) * ac), B(size_t(ldb) * bc), C(size_t(ldc) * a.n);
  fill_uniform(A, g);
  fill_uniform(B, g);
  fill_uniform(C, g);
  MapM Am(A.data(), ar, ac, Eigen::OuterStride<>(lda));
  MapM Bm(B.data(), br, bc, Eigen::OuterStride<>(ldb));
  MapM Cm(C.data(), a.m, a.n, Eigen::OuterStride<>(ldc));
  const T alpha = T(a.alpha), beta = T(a.beta);
  auto step = [&]() {
    if (beta == T(0))
      Cm.setZero();
    else if (beta != T(1))
      Cm *= beta;
    if (!tA && !tB)
      Cm.noalias() += alpha * Am * Bm;
    else if (tA && !tB)
      Cm.noalias() += alpha * Am.transpose() * Bm;
    else if (!tA && tB)
      Cm.noalias() += alpha * Am * Bm.transpose();
    else
      Cm.noalias() += alpha * Am.transpose() * Bm.transpose();
  };
  for (int i = 0; i < a.warmup; ++i) step();
  std::vector<double> ts;
  double t_all = now();
  for (int i = 0; i < a.reps; ++i) {
    double t0 = now();
    step();
    ts.push_back(now() - t0);
    if (now() - t_all > a.max_seconds) break;
  }
  std::sort(ts.begin(), ts.end());
  double med = ts[ts.size() / 2];
  double flops = 2.0 * double(a.m) * double(a.n) * double(a.k);
  int threads = 1;
#ifdef _OPENMP
  threads = omp_get_max_threads();
#endif
  double checksum = 0;
  for (long j = 0; j < a.n; ++j) checksum += double(Cm(j % a.m, j));
  std::printf(
      "{\"mode\": \"gemm\", \"dtype\": \"%c\", \"m\": %ld, \"n\": %ld, \"k\": %ld, \"ta\": \"%c\", \"tb\": \"%c\", "
      "\"reps\": %zu, \"seconds_median\": %.9g, \"seconds_min\": %.9g, \"seconds_max\": %.9g, \"gflops\": %.6g, "
      "\"threads\": %d, \"checksum\": %.17g}\n",
      a.dtype, a.m, a.n, a.k, a.ta, a.tb, ts.size(), med, ts.front(), ts.back(), flops / med * 1e-9, threads,
      checksum);
  return 0;
}

struct Problem {
  int m, n, k;
};

// Same size law as the device batch: each of m,n,k = round(exp(U[ln 3, ln 256])),
// or, with probability 0.2, all three drawn from {3,4,6,8}.
std::vector<Problem> make_batch(long count, std::mt19937_64& g) {
  std::uniform_real_distribution<double> u01(0.0, 1.0);
  std::uniform_real_distribution<double> lu(std::log(3.0), std::log(256.0));
  const int fixed[4] = {3, 4, 6, 8};
  std::vector<Problem> ps(count);
  for (auto& p : ps) {
    if (u01(g) < 0.2) {
      int s = fixed[std::min(3, int(u01(g) * 4))];
      p = {s, s, s};
    } else {
      p.m = int(std::lround(std::exp(lu(g))));
      p.n = int(std::lround(std::exp(lu(g))));
      p.k = int(std::lround(std::exp(lu(g))));
    }
  }
  return ps;
}

template <typename T, int N>
void fixed_product(const T* a, const T* b, T* c) {
  using M = Eigen::Matrix<T, N, N>;
  Eigen::Map<const M> A(a), B(b);
  Eigen::Map<M> C(c);
  C.noalias() = A * B;
}

template <typename T>
int run_batch(const Args& a) {
  using Mat = Eigen::Matrix<T, Eigen::Dynamic, Eigen::Dynamic>;
  std::mt19937_64 g(a.seed);
  std::vector<Problem> ps = make_batch(a.count, g);
  std::vector<size_t> oa(ps.size() + 1), ob(ps.size() + 1), oc(ps.size() + 1);
  oa[0] = ob[0] = oc[0] = 0;
  double flops = 0;
  for (size_t i = 0; i < ps.size(); ++i) {
    oa[i + 1] = oa[i] + size_t(ps[i].m) * ps[i].k;
    ob[i + 1] = ob[i] + size_t(ps[i].k) * ps[i].n;
    oc[i + 1] = oc[i] + size_t(ps[i].m) * ps[i].n;
    flops += 2.0 * ps[i].m * ps[i].n * double(ps[i].k);
  }
  std::vector<T> A(oa.back()), B(ob.back()), C(oc.back());
  fill_uniform(A, g);
  fill_uniform(B, g);
  auto step = [&]() {
#pragma omp parallel for schedule(dynamic, 16)
    for (long i = 0; i < long(ps.size()); ++i) {
      const Problem& p = ps[i];
      const T* pa = A.data() + oa[i];
      const T* pb = B.data() + ob[i];
      T* pc = C.data() + oc[i];
      if (p.m == p.n && p.n == p.k && (p.m == 3 || p.m == 4 || p.m == 6 || p.m == 8)) {
        switch (p.m) {
          case 3: fixed_product<T, 3>(pa, pb, pc); break;
          case 4: fixed_product<T, 4>(pa, pb, pc); break;
          case 6: fixed_product<T, 6>(pa, pb, pc); break;
          default: fixed_product<T, 8>(pa, pb, pc); break;
        }
      } else {
        Eigen::Map<const Mat> Am(pa, p.m, p.k), Bm(pb, p.k, p.n);
        Eigen::Map<Mat> Cm(pc, p.m, p.n);
        Cm.noalias() = Am * Bm;
      }
    }
  };
  for (int i = 0; i < a.warmup; ++i) step();
  std::vector<double> ts;
  double t_all = now();
  for (int i = 0; i < a.reps; ++i) {
    double t0 = now();
    step();
    ts.push_back(now() - t0);
    if (now() - t_all > a.max_seconds) break;
  }
  std::sort(ts.begin(), ts.end());
  double med = ts[ts.size() / 2];
  int threads = 1;
#ifdef _OPENMP
  threads = omp_get_max_threads();
#endif
  std::printf(
      "{\"mode\": \"batch\", \"dtype\": \"%c\", \"count\": %ld, \"reps\": %zu, \"seconds_median\": %.9g, "
      "\"seconds_min\": %.9g, \"gflops\": %.6g, \"flops\": %.6g, \"threads\": %d}\n",
      a.dtype, a.count, ts.size(), med, ts.front(), flops / med * 1e-9, flops, threads);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  Args a;
  for (int i = 1; i < argc; ++i) {
    std::string s = argv[i];
    auto val = [&](void) -> const char* {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "missing value for %s\n", s.c_str());
        std::exit(2);
      }
      return argv[++i];
    };
    if (s == "--mode") a.mode = val();
    else if (s == "--dtype") a.dtype = val()[0];
    else if (s == "--m") a.m = std::atol(val());
    else if (s == "--n") a.n = std::atol(val());
    else if (s == "--k") a.k = std::atol(val());
    else if (s == "--ta") a.ta = val()[0];
    else if (s == "--tb") a.tb = val()[0];
    else if (s == "--alpha") a.alpha = std::atof(val());
    else if (s == "--beta") a.beta = std::atof(val());
    else if (s == "--pad") a.pad = std::atol(val());
    else if (s == "--reps") a.reps = std::atoi(val());
    else if (s == "--warmup") a.warmup = std::atoi(val());
    else if (s == "--count") a.count = std::atol(val());
    else if (s == "--seed") a.seed = std::strtoull(val(), nullptr, 10);
    else if (s == "--max-seconds") a.max_seconds = std::atof(val());
    else {
      std::fprintf(stderr, "unknown argument %s\n", s.c_str());
      return 2;
    }
  }
  if (a.reps < 1) a.reps = 1;
  if (a.mode == "gemm") return a.dtype == 's' ? run_gemm<float>(a) : run_gemm<double>(a);
  if (a.mode == "batch") return a.dtype == 's' ? run_batch<float>(a) : run_batch<double>(a);
  std::fprintf(stderr, "unknown mode %s\n", a.mode.c_str());
  return 2;
}
