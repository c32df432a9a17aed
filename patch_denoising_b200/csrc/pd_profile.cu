// Launch timing registry behind pd_profile_enable / pd_profile_collect.
#include <stdio.h>
#include <string.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "pd_common.cuh"
#include "pd_profile.cuh"

namespace pd {
namespace {
struct Rec {
  std::string name;
  cudaEvent_t a, b;
};
std::mutex g_mu;
bool g_on = false;
std::vector<Rec> g_recs;
std::vector<cudaEvent_t> g_pool;
Rec g_open;
cudaEvent_t take_event() {
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

bool profile_on() { return g_on; }

void profile_begin(const char* name, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_open.name = name;
  g_open.a = take_event();
  g_open.b = take_event();
  cudaEventRecord(g_open.a, s);
}

void profile_end(cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_mu);
  cudaEventRecord(g_open.b, s);
  g_recs.push_back(g_open);
}
}  // namespace pd

extern "C" {
pd_status pd_profile_enable(int32_t on) {
  pd::g_on = on != 0;
  return PD_OK;
}

pd_status pd_profile_collect(char* buf, size_t len) {
  std::lock_guard<std::mutex> lk(pd::g_mu);
  std::map<std::string, std::pair<long, double>> agg;
  for (auto& r : pd::g_recs) {
    cudaEventSynchronize(r.b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.a, r.b);
    auto& v = agg[r.name];
    v.first += 1;
    v.second += ms;
    pd::g_pool.push_back(r.a);
    pd::g_pool.push_back(r.b);
  }
  pd::g_recs.clear();
  std::string out;
  char line[256];
  for (auto& kv : agg) {
    snprintf(line, sizeof line, "%s %ld %.6f\n", kv.first.c_str(), kv.second.first, kv.second.second);
    out += line;
  }
  if (buf && len) {
    strncpy(buf, out.c_str(), len - 1);
    buf[len - 1] = 0;
  }
  return PD_OK;
}
}
