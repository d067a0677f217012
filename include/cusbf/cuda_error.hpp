// cuda_error.hpp -- CUSBF_CUDA_CALL (drop-in for the reference's
// include/cusbf/cuda_error.hpp:11-16): throws std::runtime_error on failure.
#pragma once

#include <stdexcept>

#include <cusbf/error.hpp>

#define CUSBF_CUDA_CALL(err)                                                      \
    do {                                                                          \
        if (cudaError_t _cusbf_err = (err); _cusbf_err != cudaSuccess) {          \
            throw std::runtime_error(::cusbf::Error::cuda(_cusbf_err).message()); \
        }                                                                         \
    } while (0)
