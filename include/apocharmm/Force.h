// Force<T>: three planes of per-atom values in device memory (the
// reference's Force<T>, include/Force.h:32-140, src/Force.cu).
//
// x values are data[0 .. size), y values data[stride ..), z values
// data[2 stride ..); each plane starts on a 256-byte boundary.  Force<long
// long int> holds fixed point with 2^40 units per kcal/mol/A, the scale the
// library sums gradients in; Force<double> holds kcal/mol/A.  The values are
// gradients dU/dx, as in the reference.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "apocharmm/Check.h"

template <typename T>
class Force {
 public:
  Force() = default;
  explicit Force(const int size) { realloc(size); }
  ~Force() {
    if (m_Data) cudaFree(m_Data);
  }
  Force(const Force &) = delete;
  Force &operator=(const Force &) = delete;

  // Re-allocates for `size` atoms (contents are not kept); `fac` >= 1 leaves
  // room for growth as the reference's realloc does.
  void realloc(const int size, const float fac = 1.0f) {
    if (size < 0) throw std::invalid_argument("Force::realloc: negative size");
    const size_t per = 256 / sizeof(T);
    const int stride = (int)(((size_t)size + per - 1) / per * per);
    const size_t need = (size_t)3 * (size_t)stride;
    const size_t cap = (size_t)((double)need * (fac < 1.0f ? 1.0 : (double)fac));
    if (cap > m_Capacity || !m_Data) {
      if (m_Data) cudaFree(m_Data);
      m_Data = nullptr;
      m_Capacity = 0;
      if (cap) apocharmm_detail::cuda_check(cudaMalloc(&m_Data, cap * sizeof(T)), "Force::realloc");
      m_Capacity = cap;
    }
    m_Size = size;
    m_Stride = stride;
  }

  void clear(cudaStream_t stream = 0) {
    if (m_Data)
      apocharmm_detail::cuda_check(
          cudaMemsetAsync(m_Data, 0, (size_t)3 * m_Stride * sizeof(T), stream), "Force::clear");
  }

  int stride() const { return m_Stride; }
  int size() const { return m_Size; }
  T *xyz() { return m_Data; }
  const T *xyz() const { return m_Data; }
  T *x() { return m_Data; }
  const T *x() const { return m_Data; }
  T *y() { return m_Data + m_Stride; }
  const T *y() const { return m_Data + m_Stride; }
  T *z() { return m_Data + 2 * (size_t)m_Stride; }
  const T *z() const { return m_Data + 2 * (size_t)m_Stride; }

  // copies the three planes to the host (size() values each)
  void getXYZ(T *h_x, T *h_y, T *h_z) const {
    const size_t b = (size_t)m_Size * sizeof(T);
    apocharmm_detail::cuda_check(cudaMemcpy(h_x, x(), b, cudaMemcpyDeviceToHost), "Force::getXYZ");
    apocharmm_detail::cuda_check(cudaMemcpy(h_y, y(), b, cudaMemcpyDeviceToHost), "Force::getXYZ");
    apocharmm_detail::cuda_check(cudaMemcpy(h_z, z(), b, cudaMemcpyDeviceToHost), "Force::getXYZ");
  }
  // atom-major host copy: x0 y0 z0 x1 ...
  std::vector<T> getXYZ() const {
    std::vector<T> px(m_Size), py(m_Size), pz(m_Size), out(3 * (size_t)m_Size);
    getXYZ(px.data(), py.data(), pz.data());
    for (int i = 0; i < m_Size; ++i) {
      out[3 * (size_t)i] = px[i];
      out[3 * (size_t)i + 1] = py[i];
      out[3 * (size_t)i + 2] = pz[i];
    }
    return out;
  }

 private:
  T *m_Data = nullptr;
  size_t m_Capacity = 0;  // elements
  int m_Size = 0;
  int m_Stride = 0;
};
