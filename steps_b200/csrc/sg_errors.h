// Host-side error classes of the solver.  They mirror the reference's exception
// classes (src/steps/util/error.hpp:161-234) and are turned into sg_status codes
// at the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

namespace sg {

struct ArgErr : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct ProgErr : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct NotImplErr : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct CudaErr : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct DeviceErr : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// Sets the message returned by sg_last_error() on the calling thread.
void set_last_error(const std::string& msg);

}  // namespace sg

#define SG_CUDA(call)                                                                    \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            throw ::sg::CudaErr(std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)
