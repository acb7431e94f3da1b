// Exact betweenness on the device (see brandes.cu).
#pragma once
#include "engine.h"

namespace silvan {

// Exact betweenness of every node of G, normalised by n (n - 1) over ordered
// pairs (the quantity SILVAN estimates), into out_host[n].
int exact_betweenness(const DeviceGraph &G, double *out_host);

}  // namespace silvan
