// proposal.hpp — what the MPPI backend needs from the proposal network
// (include/mppi_b200/mppi_proposal.h) to run it inside its own closed loop.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/mppi_b200/mppi_proposal.h"

namespace mppi_b200 {

struct ProposalShape {
  uint32_t input_dim;
  uint32_t horizon;
  uint32_t control_dim;
  uint32_t out_stride;  // floats per output row
  float log_scale_min;
  float log_scale_max;
  int device;
};

ProposalShape proposal_shape(const mppi_proposal* p);

// The network's parameters as the per-agent form reads them: layer l's BF16
// weight image (K-major core-matrix layout, rows = outputs) and FP32 biases,
// the padded input width, the hidden width and the padded output count.
struct ProposalWeights {
  const uint16_t* w[4];
  const float* b[4];
  uint32_t in;
  uint32_t hidden;
  uint32_t out;
};
ProposalWeights proposal_weights(const mppi_proposal* p);

// Enqueues the network's forward pass for `rows` feature rows on `stream`
// (capturable into a CUDA graph): out[r][0..H*m) predicted u*, then m raw
// log-scales.  programmatic: launched with programmatic stream
// serialisation, so it may start while the stream's previous kernel
// finishes (it waits for that grid before it reads x).  Returns cudaSuccess
// or the launch error.
cudaError_t proposal_enqueue_forward(mppi_proposal* p, cudaStream_t stream, const float* x,
                                     uint32_t x_stride, uint32_t rows, float* out,
                                     bool programmatic = false);

// Reads and clears the device error word of the network's kernels (a
// bounded wait that gave up).  False with a message when one is set.
bool proposal_check_device_error(mppi_proposal* p, std::string* msg);

}  // namespace mppi_b200
