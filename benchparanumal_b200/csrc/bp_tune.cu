// Kernel-form autotuner for the element operators.
//
// The BP5/BP6 element operator has several forms (TMA-staged register
// pencils, line-per-thread, register pencil, tensor-core MMA; and their packed
// multi-rhs variants), each best somewhere in (degree, fields, factor storage,
// precision, lanes).  The first time a configuration is launched outside a
// stream capture, every applicable form is run on the caller's own operands --
// one untimed launch, then timed in interleaved rounds with CUDA events on the
// launch stream --
// and the fastest is kept for that configuration (and element-count class, a
// power of two) on that device; later
// launches, the captured CUDA graphs of the solvers included, use it.  While a
// stream is capturing, an untuned configuration takes the first form of its
// candidate list, the measured static choice, and is not recorded.  The
// solvers launch their operator once before capturing, so their graphs use the
// tuned form.  BP_AUTOTUNE=0 keeps the static choice everywhere.
#include <cuda_runtime.h>

#include <cstdlib>
#include <map>
#include <tuple>

#include "bp_internal.hpp"

namespace bp {
namespace {

using Key = std::tuple<int, int, int, int, int, int, int, int, int>;   // dev, kind, nq, nf, affine, bytes, lanes,
                                                                      // fused, size class
std::mutex g_lock;
std::map<Key, int> g_choice;
std::map<Key, std::vector<std::pair<int, float>>> g_times;   // measured ms per form, for reports and tests

bool autotune_enabled() {
  const char* e = getenv("BP_AUTOTUNE");
  return !(e && e[0] == '0');
}

}  // namespace

int tuned_form(const TuneConfig& c, const std::vector<int>& forms, const std::function<int(int)>& run,
               cudaStream_t s, int* form) {
  *form = forms.empty() ? -1 : forms[0];
  if (forms.size() <= 1) return BP_SUCCESS;
  int dev = 0;
  BP_TRY(current_device(&dev));
  const Key key{dev, c.kind, c.nq, c.nf, c.affine, c.bytes, c.lanes, c.fused, c.ecls};
  {
    std::lock_guard<std::mutex> lock(g_lock);
    auto it = g_choice.find(key);
    if (it != g_choice.end()) {
      *form = it->second;
      return BP_SUCCESS;
    }
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  BP_CUDA_TRY(cudaStreamIsCapturing(s, &cap));
  if (cap != cudaStreamCaptureStatusNone) return BP_SUCCESS;   // the static choice, not recorded
  if (!autotune_enabled()) {
    std::lock_guard<std::mutex> lock(g_lock);
    g_choice[key] = forms[0];
    return BP_SUCCESS;
  }
  // Every applicable form first runs once untimed (this also finds the forms
  // that do not cover the configuration), then kRounds rounds time each form
  // over two launches in turn, and a form's time is its fastest round: forms
  // interleaved in time see the same clocks and L2 state (timing them one
  // after the other favoured whichever ran once the clocks had ramped up), and
  // the minimum drops rounds disturbed by anything else on the device.  The
  // static choice (the list's first form) is kept unless another is faster
  // by more than kMargin.
  constexpr int kRounds = 3, kLaunches = 2;
  constexpr float kMargin = 0.02f;
  std::vector<int> live;
  int rc = BP_SUCCESS;
  for (int f : forms) {
    rc = run(f);
    if (rc == 1) {
      rc = BP_SUCCESS;
      continue;
    }
    if (rc != BP_SUCCESS) return rc;
    live.push_back(f);
  }
  if (live.empty()) return fail(BP_ERROR_ARG, "element operator: no kernel form covers this configuration");
  cudaEvent_t e0, e1;
  BP_CUDA_TRY(cudaEventCreate(&e0));
  BP_CUDA_TRY(cudaEventCreate(&e1));
  std::vector<float> best_of(live.size(), 0.f);
  for (int round = 0; round < kRounds && rc == BP_SUCCESS; ++round) {
    for (size_t i = 0; i < live.size() && rc == BP_SUCCESS; ++i) {
      cudaEventRecord(e0, s);
      for (int k = 0; k < kLaunches && rc == BP_SUCCESS; ++k) rc = run(live[i]);
      cudaEventRecord(e1, s);
      if (rc != BP_SUCCESS) break;
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        rc = cuda_fail(cudaGetLastError(), "cudaEventSynchronize", __FILE__, __LINE__);
        break;
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      ms /= (float)kLaunches;
      if (round == 0 || ms < best_of[i]) best_of[i] = ms;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  BP_TRY(rc);
  std::vector<std::pair<int, float>> times;
  size_t bi = 0;
  for (size_t i = 0; i < live.size(); ++i) {
    times.push_back({live[i], best_of[i]});
    if (best_of[i] < best_of[bi]) bi = i;
  }
  // the static choice stands unless beaten by more than the margin
  if (live[0] == forms[0] && best_of[bi] > (1.f - kMargin) * best_of[0]) bi = 0;
  const int best = live[bi];
  *form = best;
  std::lock_guard<std::mutex> lock(g_lock);
  g_choice[key] = best;
  g_times[key] = times;
  return BP_SUCCESS;
}

int tuned_report(const TuneConfig& c, int* form, int* nforms, int* forms, float* ms, int cap) {
  int dev = 0;
  BP_TRY(current_device(&dev));
  const Key key{dev, c.kind, c.nq, c.nf, c.affine, c.bytes, c.lanes, c.fused, c.ecls};
  std::lock_guard<std::mutex> lock(g_lock);
  auto it = g_choice.find(key);
  *form = it == g_choice.end() ? -1 : it->second;
  *nforms = 0;
  auto jt = g_times.find(key);
  if (jt != g_times.end())
    for (const auto& t : jt->second)
      if (*nforms < cap) {
        forms[*nforms] = t.first;
        ms[*nforms] = t.second;
        ++*nforms;
      }
  return BP_SUCCESS;
}

void tuned_clear() {
  std::lock_guard<std::mutex> lock(g_lock);
  g_choice.clear();
  g_times.clear();
}

}  // namespace bp
