// Estimation server (continuous batching), see server.cu.
#pragma once
#include <cstdint>
#include <vector>

#include "graph_host.h"
#include "silvan.h"

namespace silvan {

struct Server;
int server_create(uint64_t n_max, uint64_t budget, uint32_t slots, Server **out);
int server_submit(Server *s, const HostGraph &h, const std::vector<uint32_t> &cc, uint32_t ncomp,
                  uint32_t diameter, const silvan_params_t &p, uint64_t *id);
int server_poll(Server *s, uint64_t id, int32_t *state, silvan_result_t *res, double *latency,
                double *queue_s);
int server_wait(Server *s, uint64_t id, double timeout_s);
int server_estimates(Server *s, uint64_t id, double *out, uint32_t n, uint32_t *topk_nodes,
                     double *topk_values, uint32_t topk_cap, uint32_t *topk_count);
int server_stats(Server *s, silvan_server_stats_t *st);
void server_destroy(Server *s);

}  // namespace silvan
