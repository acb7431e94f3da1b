// Device-side edge-list ingest (see ingest.cu).
#pragma once
#include <string>

#include "engine.h"

namespace silvan {

// Reads a `u v` edge list with the reference loader's semantics and builds
// the CSR on the device; fills G (device arrays, the host copy, components
// and diameter bound).  Returns 0 or a negative SILVAN_E_* code, with a
// message in err for file and parse errors.
int device_ingest(const char *path, bool directed, DeviceGraph &G, std::string &err);

}  // namespace silvan
