// Thin C entry points over the reference's own host code, compiled from the
// reference sources where they lie (include path set by oracle/build_ref.py).
// TEST INFRASTRUCTURE ONLY: used to pin the oracle and as the timed
// reference CPU arm; never linked into the product.
//   Matrix<T>::operator*   -- Kernel/cuda/src/Matrix.h:183-201
//   Matrix<T>::fillRandom  -- Kernel/cuda/src/Matrix.h:75-87 (mt19937(seed), U[0,1))
#include "Matrix.h"
#include <cstring>

template <class T>
static void product(int m, int n, int k, const T* A, const T* B, T* C) {
  Matrix<T> a(m, k), b(k, n);
  std::memcpy(a.elems, A, sizeof(T) * (size_t)m * k);
  std::memcpy(b.elems, B, sizeof(T) * (size_t)k * n);
  Matrix<T> c = a * b;
  std::memcpy(C, c.elems, sizeof(T) * (size_t)m * n);
}

extern "C" void ref_cpu_gemm_f64(int m, int n, int k, const double* A, const double* B, double* C) {
  product<double>(m, n, k, A, B, C);
}
extern "C" void ref_cpu_gemm_f32(int m, int n, int k, const float* A, const float* B, float* C) {
  product<float>(m, n, k, A, B, C);
}
// Timed reference CPU arm: B is copied once into a Matrix<double>; each call
// multiplies a slab of A rows with it through Matrix<double>::operator*.
static Matrix<double>* g_b = nullptr;
extern "C" void ref_cpu_set_b(int k, int n, const double* B) {
  delete g_b;
  g_b = new Matrix<double>(k, n);
  std::memcpy(g_b->elems, B, sizeof(double) * (size_t)k * n);
}
extern "C" void ref_cpu_rows(int rows, int k, const double* A_rows, double* C_rows) {
  Matrix<double> a(rows, k);
  std::memcpy(a.elems, A_rows, sizeof(double) * (size_t)rows * k);
  Matrix<double> c = a * (*g_b);
  std::memcpy(C_rows, c.elems, sizeof(double) * (size_t)rows * g_b->cols);
}

extern "C" void ref_fill_random_f32(int seed, int rows, int cols, float* out) {
  Matrix<float> x(rows, cols);
  x.fillRandom(seed);
  std::memcpy(out, x.elems, sizeof(float) * (size_t)rows * cols);
}
extern "C" void ref_fill_random_f64(int seed, int rows, int cols, double* out) {
  Matrix<double> x(rows, cols);
  x.fillRandom(seed);
  std::memcpy(out, x.elems, sizeof(double) * (size_t)rows * cols);
}
