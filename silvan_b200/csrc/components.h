// Components and diameter bound of an undirected graph on the device (see
// components.cu).
#pragma once
#include "engine.h"

namespace silvan {

// Fills G.d_cc (component ids in the reference's numbering), G.ncomp and
// G.diameter from the device CSR of an undirected graph.
int device_undirected_components(DeviceGraph &G, cudaStream_t stream);

// G.diameter of a directed graph from its device CSR and G.d_cc / G.ncomp
// (component ids in the reference's Tarjan numbering): the pivots, their
// eccentricities inside their components and the AllCCUpperBound recursion
// (silvan/src/Graph.cpp:205-316), on the device.
int device_directed_bound(DeviceGraph &G, cudaStream_t stream);

}  // namespace silvan
