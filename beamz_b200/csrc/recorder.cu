// Time-domain field recorders: after a step, the chosen components (whole
// arrays, or interpolated plane / line samples) are written into the next
// record slot (beamz/simulation/observe.py:588-646 _record_fields;
// beamz/devices/monitors/compiler.py:286-412 FieldRecorder).
//
// One launch per recorder and step; the device step counter decides whether
// the step records (the host never reads it), so the launch can sit in a
// captured graph.  Every block reads the record count from the slot of the
// step's parity and block 0 writes the next count into the other slot, so no
// block can see a count updated by this launch.

#include "kernels.cuh"

namespace fdtd {

namespace {

constexpr int kRecThreads = 256;

__global__ void __launch_bounds__(kRecThreads) record_kernel(RecorderDev r, const int* counter, int step_offset) {
  const int step = counter[0] + step_offset;
  const bool hit = (step + 1) % r.interval == 0;
  const int n = r.count[step & 1];
  const bool rec = hit && n < r.capacity;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    r.count[(step + 1) & 1] = n + (rec ? 1 : 0);
    if (rec) {
      r.steps[n] = step + 1;
      r.times[n] = r.step_time[step < r.step_time_len ? step : r.step_time_len - 1];
    }
  }
  if (!rec) return;
  const int64_t total = r.start[r.ncomp];
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * kRecThreads + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * kRecThreads) {
    int q = 0;
    while (q + 1 < r.ncomp && t >= r.start[q + 1]) ++q;
    const int64_t v = t - r.start[q];
    const int64_t V = r.start[q + 1] - r.start[q];
    const float* f = r.field[q];
    float x = 0.0f;
    if (r.slots[q] == 0) {  // whole component, its own (z, y, x) order
      const int64_t i = v % r.dx[q];
      const int64_t rest = v / r.dx[q];
      const int64_t j = rest % r.dy[q], k = rest / r.dy[q];
      x = f[k * r.plane[q] + j * r.row[q] + i];
    } else {
      for (int s = 0; s < r.slots[q]; ++s) {
        const float w = r.w[q][s * V + v];
        if (w == 0.0f) break;
        const int o = r.idx[q][s * V + v];
        if (o >= 0 && o < r.field_len[q]) x = x + f[o] * w;
      }
    }
    r.values[q][static_cast<int64_t>(n) * V + v] = x * r.sign[q];
  }
}

}  // namespace

cudaError_t launch_record(cudaStream_t s, const RecorderDev& r, const int* counter, int step_offset) {
  const int64_t total = r.start[r.ncomp];
  int64_t blocks = (total + kRecThreads - 1) / kRecThreads;
  if (blocks < 1) blocks = 1;
  if (blocks > 8 * 148) blocks = 8 * 148;
  record_kernel<<<static_cast<unsigned>(blocks), kRecThreads, 0, s>>>(r, counter, step_offset);
  return cudaPeekAtLastError();
}

}  // namespace fdtd
