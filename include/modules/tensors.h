// Container types of the LaughlinEdge API: vector<T>, cmatrix<T> (complex
// matrix, row-major) and rank3tensor<T>.  Drop-in for the subset of the
// reference's modules/tensors.h that the public API exchanges (sector lists,
// the metric passed to occupation_numbers_compute, returned matrices).
#ifndef LAUGHLINEDGE_TENSORS_H
#define LAUGHLINEDGE_TENSORS_H

#include <cstddef>
#include <initializer_list>
#include <vector>

#include "complex_numbers.h"

template <typename T>
class vector {
 public:
  vector() = default;
  explicit vector(int n) : v_(n) {}
  vector(int n, const T& x0) : v_(n, x0) {}
  vector(std::initializer_list<T> l) : v_(l) {}
  T& operator[](int i) { return v_[i]; }
  const T& operator[](int i) const { return v_[i]; }
  int size() const { return int(v_.size()); }
  T* vec_pointer() { return v_.data(); }
  const T* vec_pointer() const { return v_.data(); }
  void push_back(const T& x) { v_.push_back(x); }
  T* begin() { return v_.data(); }
  T* end() { return v_.data() + v_.size(); }
  const T* begin() const { return v_.data(); }
  const T* end() const { return v_.data() + v_.size(); }

 private:
  std::vector<T> v_;
};

template <typename T>
class cmatrix {
 public:
  cmatrix() = default;
  cmatrix(int r, int c) : r_(r), c_(c), a_(size_t(r) * c) {}
  cmatrix(int r, int c, const complex<T>& x0) : r_(r), c_(c), a_(size_t(r) * c, x0) {}
  complex<T>& operator()(int i, int j) { return a_[size_t(i) * c_ + j]; }
  const complex<T>& operator()(int i, int j) const { return a_[size_t(i) * c_ + j]; }
  int rows() const { return r_; }
  int cols() const { return c_; }
  complex<T>* data() { return a_.data(); }
  const complex<T>* data() const { return a_.data(); }
  cmatrix adjoint() const {
    cmatrix t(c_, r_);
    for (int i = 0; i < r_; ++i)
      for (int j = 0; j < c_; ++j) t(j, i) = conj((*this)(i, j));
    return t;
  }
  friend cmatrix operator+(const cmatrix& a, const cmatrix& b) {
    cmatrix t(a.r_, a.c_);
    for (size_t k = 0; k < a.a_.size(); ++k) t.a_[k] = a.a_[k] + b.a_[k];
    return t;
  }
  friend cmatrix operator/(const cmatrix& a, T s) {
    cmatrix t(a.r_, a.c_);
    for (size_t k = 0; k < a.a_.size(); ++k) t.a_[k] = a.a_[k] / s;
    return t;
  }

 private:
  int r_ = 0, c_ = 0;
  std::vector<complex<T>> a_;
};

template <typename T>
class rank3tensor {
 public:
  rank3tensor() = default;
  rank3tensor(int a, int b, int c) : s1_(a), s2_(b), s3_(c), v_(size_t(a) * b * c) {}
  rank3tensor(int a, int b, int c, const T& x0) : s1_(a), s2_(b), s3_(c), v_(size_t(a) * b * c, x0) {}
  T& operator()(int i, int j, int k) { return v_[(size_t(i) * s2_ + j) * s3_ + k]; }
  const T& operator()(int i, int j, int k) const { return v_[(size_t(i) * s2_ + j) * s3_ + k]; }
  int s1() const { return s1_; }
  int s2() const { return s2_; }
  int s3() const { return s3_; }

 private:
  int s1_ = 0, s2_ = 0, s3_ = 0;
  std::vector<T> v_;
};

#endif
