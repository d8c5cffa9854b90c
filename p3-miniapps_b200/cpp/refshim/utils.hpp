// Reference-facing C++ layer: miniapps/vlp4d/thrust/utils.hpp:1-22.
#ifndef VLP4D_B200_REFSHIM_UTILS_HPP
#define VLP4D_B200_REFSHIM_UTILS_HPP

#include <cuda_runtime.h>

#define DISALLOW_COPY_AND_ASSIGN(ClassName) \
  ClassName(const ClassName &);             \
  void operator=(const ClassName &);

// The reference synchronises the device after every stage of a step.
inline void synchronize() { cudaDeviceSynchronize(); }

#endif
