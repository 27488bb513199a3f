// Seeded Gaussian sketches generated on the device (libstdc++ mt19937 +
// normal_distribution<double> streams, column-major fill).
#pragma once

#include "common.cuh"

namespace fpls {

// nstreams independent streams: stream s (seed d_seeds[s], device array)
// writes len values at out + s * ld.
void device_gaussian_streams(double* out, long long len, long long ld, const unsigned int* d_seeds, int nstreams,
                             cudaStream_t stream);

// One stream of n_elem values (a rows x cols column-major sketch).
void device_gaussian(double* out, long long n_elem, unsigned int seed);

}  // namespace fpls
