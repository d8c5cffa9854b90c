// Reference-facing C++ layer over libvlp4d_b200: the types of the reference's
// single-process CUDA variant (miniapps/vlp4d/thrust/types.hpp:10-58), with
// the same names and meanings, backed by device memory and the C ABI in
// include/vlp4d_b200.h.  Together with config.hpp, efield.hpp, diags.hpp,
// field.hpp, advection.hpp, init.hpp and utils.hpp in this directory, the
// reference's own vlp4d.cpp and timestep.hpp compile unchanged against it.
#ifndef VLP4D_B200_REFSHIM_TYPES_HPP
#define VLP4D_B200_REFSHIM_TYPES_HPP

#include <cuda_runtime.h>

#include <array>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../../include/vlp4d_b200.h"

using float32 = float;
using float64 = double;
using Real = float64;

template <size_t ND>
using shape_nd = std::array<int, ND>;

namespace vlp4d_shim {

// Non-zero status from the C ABI -> exception with the library's message.
// (The reference exits the process on CUDA errors, lib/Cuda_Helper.hpp:8-16;
// an exception lets the caller decide.)
inline void check(int rc, const char *what) {
  if (rc != VLP4D_OK) throw std::runtime_error(std::string(what) + ": " + vlp4d_last_error());
}

// Owning device array of `Real` in layout_left order with an optional host
// mirror, standing in for the reference's View (lib/thrust/View.hpp:29-319):
// data() is the device pointer the kernels use, operator() indexes the host
// mirror, updateDevice()/updateSelf() copy between them.
template <size_t ND>
class DeviceView {
 public:
  using value_type = Real;

  DeviceView() = default;
  template <typename... I>
  explicit DeviceView(const std::string &name, I... extents) : name_(name), ext_{static_cast<size_t>(extents)...} {
    static_assert(sizeof...(I) == ND, "one extent per dimension");
    allocate();
  }
  DeviceView(const std::string &name, const shape_nd<ND> &extents) : name_(name) {
    for (size_t i = 0; i < ND; ++i) ext_[i] = static_cast<size_t>(extents[i]);
    allocate();
  }
  // A non-owning view of memory owned elsewhere (the context's 2D fields).
  static DeviceView wrap(const std::string &name, Real *dev, const shape_nd<ND> &extents) {
    DeviceView v;
    v.name_ = name;
    for (size_t i = 0; i < ND; ++i) v.ext_[i] = static_cast<size_t>(extents[i]);
    v.size_ = 1;
    for (size_t e : v.ext_) v.size_ *= e;
    v.dev_ = dev;
    v.owned_ = false;
    v.host_.assign(v.size_, 0.0);
    return v;
  }
  ~DeviceView() { release(); }
  DeviceView(const DeviceView &) = delete;
  DeviceView &operator=(const DeviceView &) = delete;
  DeviceView(DeviceView &&o) noexcept { *this = std::move(o); }
  DeviceView &operator=(DeviceView &&o) noexcept {
    if (this != &o) {
      release();
      name_ = std::move(o.name_);
      ext_ = o.ext_;
      size_ = o.size_;
      dev_ = o.dev_;
      owned_ = o.owned_;
      host_ = std::move(o.host_);
      o.dev_ = nullptr;
      o.size_ = 0;
      o.owned_ = false;
    }
    return *this;
  }

  Real *data() const { return dev_; }
  size_t size() const { return size_; }
  size_t extent(size_t r) const { return ext_[r]; }
  const std::string &name() const { return name_; }

  void updateDevice() {
    check(cudaMemcpy(dev_, host_.data(), size_ * sizeof(Real), cudaMemcpyHostToDevice) == cudaSuccess
              ? VLP4D_OK : VLP4D_ERR_CUDA, "updateDevice");
  }
  void updateSelf() {
    check(cudaMemcpy(host_.data(), dev_, size_ * sizeof(Real), cudaMemcpyDeviceToHost) == cudaSuccess
              ? VLP4D_OK : VLP4D_ERR_CUDA, "updateSelf");
  }
  template <typename... I>
  Real &operator()(I... idx) {
    static_assert(sizeof...(I) == ND, "one index per dimension");
    const size_t ids[ND] = {static_cast<size_t>(idx)...};
    size_t off = 0, stride = 1;
    for (size_t i = 0; i < ND; ++i) {
      off += ids[i] * stride;
      stride *= ext_[i];
    }
    return host_[off];
  }
  void swap(DeviceView &o) { std::swap(*this, o); }

 private:
  void allocate() {
    size_ = 1;
    for (size_t e : ext_) size_ *= e;
    void *p = nullptr;
    if (cudaMalloc(&p, size_ * sizeof(Real)) != cudaSuccess) throw std::runtime_error("cudaMalloc " + name_);
    dev_ = static_cast<Real *>(p);
    owned_ = true;
    host_.assign(size_, 0.0);
  }
  void release() {
    if (owned_ && dev_) cudaFree(dev_);
    dev_ = nullptr;
    owned_ = false;
  }

  std::string name_;
  std::array<size_t, ND> ext_{};
  size_t size_ = 0;
  Real *dev_ = nullptr;
  bool owned_ = false;
  std::vector<Real> host_;
};

}  // namespace vlp4d_shim

using RealView1D = vlp4d_shim::DeviceView<1>;
using RealView2D = vlp4d_shim::DeviceView<2>;
using RealView4D = vlp4d_shim::DeviceView<4>;

#endif
