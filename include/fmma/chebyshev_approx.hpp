// fmma/chebyshev_approx.hpp — header-only drop-in for fockl/FMMA's
// fmma::CHEBYSHEV_APPROX<TYPE,DIM> (reference include/fmma/chebyshev_approx.hpp
// and src/chebyshev_approx.cpp:36-101), fitting and evaluating on a B200
// through the C ABI of fmma_b200.h.
//
// Kept: the public members Nth, fn (default |x|^2), coef and size,
// initialize() and predict(pos), the node and coefficient order (dimension 0
// fastest) and the reference's error behaviour (message on stderr,
// exit(EXIT_FAILURE), e.g. for a point outside [-1, 1]).  fn is a host
// callable evaluated on the host at the (Nth+1)^DIM nodes, as in the
// reference; the coefficients are the exact solution of the reference's
// collocation system (the reference stops its GCR iteration at a squared
// residual of 1e-6), computed on the device.  Extension: predict over a
// vector of points in one launch.
#pragma once

#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <string>
#include <vector>

#include "../fmma_b200.h"

namespace fmma {

template <typename TYPE, std::size_t DIM>
class CHEBYSHEV_APPROX {
 public:
  using point = std::array<TYPE, DIM>;
  int Nth = 0;
  std::function<TYPE(const point& pos)> fn = [](const point& pos) {
    double len2 = 0.0;
    for (std::size_t dim = 0; dim < DIM; ++dim) len2 += pos[dim] * pos[dim];
    return (TYPE)len2;
  };
  std::vector<TYPE> coef;
  std::size_t size = 0;

  CHEBYSHEV_APPROX() = default;
  ~CHEBYSHEV_APPROX() {
    if (ctx_) fmma_ctx_destroy(ctx_);
  }
  CHEBYSHEV_APPROX(const CHEBYSHEV_APPROX&) = delete;
  CHEBYSHEV_APPROX& operator=(const CHEBYSHEV_APPROX&) = delete;

  void set_device(int d) { device_ = d; }

  void initialize() {
    size = 1;
    for (std::size_t i = 0; i < DIM; ++i) size *= (std::size_t)(Nth + 1);
    std::vector<double> node((std::size_t)Nth + 1);
    check(fmma_cheb_nodes(Nth, node.data()));
    std::vector<double> values(size), c(size);
    const std::size_t n = (std::size_t)Nth + 1;
    for (std::size_t i = 0; i < size; ++i) {
      point pos;
      std::size_t ic = i;
      for (std::size_t q = 0; q < DIM; ++q) {  // dimension 0 fastest
        pos[q] = (TYPE)node[ic % n];
        ic /= n;
      }
      values[i] = (double)fn(pos);
    }
    check(fmma_cheb_fit_d(context(), (int)DIM, Nth, 1, values.data(), c.data(), FMMA_MEM_HOST));
    coef.assign(c.begin(), c.end());
  }

  TYPE predict(const point& pos) {
    std::vector<TYPE> out;
    predict(std::vector<point>{pos}, out);
    return out[0];
  }

  // every point in one launch (extension)
  void predict(const std::vector<point>& pos, std::vector<TYPE>& out) {
    if (coef.size() != size || size == 0) fail("CHEBYSHEV_APPROX: initialize() first (coef size != size)");
    std::vector<double> c(coef.begin(), coef.end()), p(pos.size() * DIM), o(pos.size());
    for (std::size_t i = 0; i < pos.size(); ++i)
      for (std::size_t q = 0; q < DIM; ++q) p[i * DIM + q] = (double)pos[i][q];
    check(fmma_cheb_eval_d(context(), (int)DIM, Nth, 1, c.data(), (int64_t)pos.size(), p.data(), o.data(),
                           FMMA_MEM_HOST));
    out.assign(o.begin(), o.end());
  }

 private:
  [[noreturn]] void fail(const std::string& msg) {
    std::fprintf(stderr, "%s:%d ERROR : %s\n", __FILE__, __LINE__, msg.c_str());
    std::exit(EXIT_FAILURE);
  }
  void check(fmma_status st) {
    if (st != FMMA_OK) fail(fmma_last_error());
  }
  fmma_ctx* context() {
    if (!ctx_) check(fmma_ctx_create(device_, &ctx_));
    return ctx_;
  }
  fmma_ctx* ctx_ = nullptr;
  int device_ = 0;
};

}  // namespace fmma
