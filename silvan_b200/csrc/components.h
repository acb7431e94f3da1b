// Components and diameter bound of an undirected graph on the device (see
// components.cu).
#pragma once
#include "engine.h"

namespace silvan {

// Fills G.d_cc (component ids in the reference's numbering), G.ncomp and
// G.diameter from the device CSR of an undirected graph.
int device_undirected_components(DeviceGraph &G, cudaStream_t stream);

}  // namespace silvan
