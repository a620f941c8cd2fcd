// tensor_contraction.cpp -- double-precision contractions of Eigen's Tensor module running on
// libeigen_b200.so.
//
// Compiled against the reference's unsupported/Eigen/Tensor with
// eigen_b200/eigen_tensor_contraction.h, which specialises the contraction's blocking and
// kernel (the customisation point of TensorContraction.h:128-157) for double so that each
// contraction is one dgemm_ call into the library.  The program contracts tensors of rank
// 2..4 over one or two index pairs, on the default device and on a thread pool, checks each
// result against a direct loop in long double, and prints one JSON line with the errors and
// the library's dgemm_ call count.  Exit status 0 when every check passes.
// With arguments "time S K [threads]" it times C(S, S) = A(S, K1, K2) . B(K1, K2, S) instead.
#define EIGEN_USE_THREADS
#include <unsupported/Eigen/Tensor>

// Built twice: with the library's kernel, and with EIGEN_TENSOR_STOCK_CONTRACTION as Eigen's
// own contraction (timing comparison only).
#ifndef EIGEN_TENSOR_STOCK_CONTRACTION
#include "eigen_b200/eigen_tensor_contraction.h"
#endif

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

using Eigen::Index;
using Pair = Eigen::IndexPair<Index>;

template <int NA, int NB, int NC, size_t P>
double check(const Eigen::Tensor<double, NA>& A, const Eigen::Tensor<double, NB>& B,
             const Eigen::array<Pair, P>& dims, const Eigen::Tensor<double, NC>& C) {
  // direct evaluation over every index of A and B
  Eigen::Tensor<long double, NC> R(C.dimensions());
  R.setZero();
  Eigen::array<Index, NA> ia;
  Eigen::array<Index, NB> ib;
  const Index na = A.size(), nb = B.size();
  for (Index x = 0; x < na; ++x) {
    Index t = x;
    for (int d = 0; d < NA; ++d) {
      ia[d] = t % A.dimension(d);
      t /= A.dimension(d);
    }
    for (Index y = 0; y < nb; ++y) {
      Index u = y;
      for (int d = 0; d < NB; ++d) {
        ib[d] = u % B.dimension(d);
        u /= B.dimension(d);
      }
      bool match = true;
      for (size_t p = 0; p < P; ++p) match = match && ia[dims[p].first] == ib[dims[p].second];
      if (!match) continue;
      Eigen::array<Index, NC> ic;
      int c = 0;
      for (int d = 0; d < NA; ++d) {
        bool contracted = false;
        for (size_t p = 0; p < P; ++p) contracted = contracted || dims[p].first == d;
        if (!contracted) ic[c++] = ia[d];
      }
      for (int d = 0; d < NB; ++d) {
        bool contracted = false;
        for (size_t p = 0; p < P; ++p) contracted = contracted || dims[p].second == d;
        if (!contracted) ic[c++] = ib[d];
      }
      R(ic) += (long double)A(ia) * (long double)B(ib);
    }
  }
  long double num = 0, den = 0;
  for (Index i = 0; i < C.size(); ++i) {
    const long double d = (long double)C.data()[i] - R.data()[i];
    num += d * d;
    den += R.data()[i] * R.data()[i];
  }
  return double(std::sqrt(num / den));
}

double time_contraction(Index S, Index K, int threads) {
  Eigen::Tensor<double, 3> A(S, K, K), B(K, K, S);
  A.setRandom();
  B.setRandom();
  Eigen::Tensor<double, 2> C(S, S);
  const Eigen::array<Pair, 2> dims = {Pair(1, 0), Pair(2, 1)};
  Eigen::ThreadPool pool(threads);
  Eigen::ThreadPoolDevice dev(&pool, threads);
  double best = 1e30;
  for (int r = 0; r < 3; ++r) {
    const auto t0 = std::chrono::steady_clock::now();
    if (threads > 1)
      C.device(dev) = A.contract(B, dims);
    else
      C = A.contract(B, dims);
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    best = std::min(best, s);
  }
  return best;
}

int main(int argc, char** argv) {
  if (argc > 1 && std::strcmp(argv[1], "time") == 0) {
    const Index S = argc > 2 ? std::atoi(argv[2]) : 2048, K = argc > 3 ? std::atoi(argv[3]) : 64;
    const int threads = argc > 4 ? std::atoi(argv[4]) : 1;
    const double s = time_contraction(S, K, threads);
#ifdef EIGEN_TENSOR_STOCK_CONTRACTION
    const char* path = "Eigen's own contraction kernel";
#else
    const char* path = "libeigen_b200";
#endif
    std::printf("{\"m\": %ld, \"n\": %ld, \"k\": %ld, \"threads\": %d, \"kernel\": \"%s\", \"s\": %.4f, "
                "\"tflops\": %.4f}\n",
                long(S), long(S), long(K * K), threads, path, s, 2.0 * S * S * K * K / s / 1e12);
    return 0;
  }
#ifdef EIGEN_TENSOR_STOCK_CONTRACTION
  return 2;  // the stock build only times
#else
  std::srand(3);
  double worst = 0;
  {  // a matrix product written as a contraction
    Eigen::Tensor<double, 2> A(130, 70), B(70, 90);
    A.setRandom();
    B.setRandom();
    const Eigen::array<Pair, 1> dims = {Pair(1, 0)};
    Eigen::Tensor<double, 2> C = A.contract(B, dims);
    worst = std::max(worst, check(A, B, dims, C));
  }
  {  // rank 3 x rank 3 over two index pairs, contracted dimensions not leading
    Eigen::Tensor<double, 3> A(40, 12, 9), B(9, 12, 33);
    A.setRandom();
    B.setRandom();
    const Eigen::array<Pair, 2> dims = {Pair(1, 1), Pair(2, 0)};
    Eigen::Tensor<double, 2> C = A.contract(B, dims);
    worst = std::max(worst, check(A, B, dims, C));
  }
  {  // rank 4 x rank 3, result of rank 3, on a thread pool
    Eigen::Tensor<double, 4> A(16, 7, 11, 6);
    Eigen::Tensor<double, 3> B(11, 25, 7);
    A.setRandom();
    B.setRandom();
    const Eigen::array<Pair, 2> dims = {Pair(1, 2), Pair(2, 0)};
    Eigen::ThreadPool pool(4);
    Eigen::ThreadPoolDevice dev(&pool, 4);
    Eigen::Tensor<double, 3> C(16, 6, 25);
    C.device(dev) = A.contract(B, dims);
    worst = std::max(worst, check(A, B, dims, C));
  }
  {  // a contraction inside a larger expression
    Eigen::Tensor<double, 2> A(64, 48), B(48, 32), D(64, 32);
    A.setRandom();
    B.setRandom();
    D.setRandom();
    const Eigen::array<Pair, 1> dims = {Pair(1, 0)};
    Eigen::Tensor<double, 2> C = A.contract(B, dims) * 2.0 + D;
    Eigen::Tensor<double, 2> P = A.contract(B, dims);
    Eigen::Tensor<double, 2> W = P * 2.0 + D;
    Eigen::Tensor<double, 0> diff = (C - W).abs().maximum();
    worst = std::max(worst, check(A, B, dims, P));
    worst = std::max(worst, double(diff()));
  }
  const long long calls = eb2_routine_calls("dgemm");
  std::printf("{\"worst_rel_err\": %.3e, \"dgemm_calls\": %lld, \"last_error\": %d}\n", worst, calls,
              eb2_last_error());
  return (worst < 1e-14 && calls >= 5 && eb2_last_error() == 0) ? 0 : 1;
#endif
}
