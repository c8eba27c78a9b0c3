// hg_autosave.cu -- restart files written while the solver keeps stepping.
//
// The reference's time loop stops every `Autosave interval` iterations to write Storage%Q
// (Solver/src/Approximation/DGTimeIntegrator.f90:216-218 -> TimeIntegrator_Autosave :413-454).  Here
// the state is copied on the context's stream into pinned host memory (ordered after the launches
// already queued, so it is the state of the requested iteration) and a host thread writes the
// NetCDF file once that copy has completed; the caller goes on queueing steps meanwhile.  A
// composite context (mixed orders) copies each part and the thread restores Storage%Q's element
// order before writing.
#include "hg_ctx.h"

#include <cstring>
#include <thread>

extern "C" int hg_write_restart(const char* path, double t, int32_t iter, const double* Q, int64_t ndof, int32_t N,
                                int32_t n_elements);
extern "C" const char* hg_restart_last_error(void);

struct AutosaveJob {
  std::thread th;
  cudaEvent_t done = nullptr;
  std::vector<double*> pinned;     // one buffer (or one per part)
  std::vector<size_t> count;
  std::vector<double> order;       // host staging in Storage%Q order (composite)
  std::string err;
  bool busy = false;
  ~AutosaveJob() {
    if (th.joinable()) th.join();
    for (double* p : pinned) if (p) cudaFreeHost(p);
    if (done) cudaEventDestroy(done);
  }
};

void autosave_finish(hg_ctx* c) {
  if (c->autosave && c->autosave->th.joinable()) c->autosave->th.join();
  if (c->autosave) c->autosave->busy = false;
}

static int fail_ctx(hg_ctx* c, const std::string& msg) {
  c->err = msg;
  return 1;
}

extern "C" int hg_save_restart_async(hg_ctx* c, const char* path, double t, int32_t iter) {
  if (!c || !path) return 1;
  try {
    if (!c->state_set) throw std::runtime_error("state not set (call hg_set_state first)");
    autosave_finish(c);   // one write in flight: its buffers are reused
    if (!c->autosave) {
      c->autosave = std::make_shared<AutosaveJob>();
      HG_CUDA(cudaEventCreateWithFlags(&c->autosave->done, cudaEventDisableTiming));
    }
    AutosaveJob& j = *c->autosave;
    j.err.clear();
    std::vector<hg_ctx*> src = c->parts.empty() ? std::vector<hg_ctx*>{c} : c->parts;
    if (j.pinned.size() != src.size()) {
      for (double* p : j.pinned) if (p) cudaFreeHost(p);
      j.pinned.assign(src.size(), nullptr);
      j.count.assign(src.size(), 0);
    }
    for (size_t k = 0; k < src.size(); ++k) {
      const size_t n = size_t(src[k]->ndof);
      if (j.count[k] != n) {
        if (j.pinned[k]) cudaFreeHost(j.pinned[k]);
        j.pinned[k] = nullptr;
        HG_CUDA(cudaMallocHost(reinterpret_cast<void**>(&j.pinned[k]), n * sizeof(double)));
        j.count[k] = n;
      }
      HG_CUDA(cudaMemcpyAsync(j.pinned[k], src[k]->d_Q, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    HG_CUDA(cudaEventRecord(j.done, c->stream));
    const std::string file(path);
    const int N = c->N, E = c->n_el;
    const int64_t ndof = c->ndof;
    const bool composite = !c->parts.empty();
    // element maps of a composite, copied for the thread (the context may change them meanwhile only
    // through calls that first finish this write)
    std::vector<int> el_part = c->el_part, el_local = c->el_local, el_N = c->el_N;
    std::vector<int64_t> el_offset = c->el_offset;
    j.busy = true;
    AutosaveJob* jp = &j;
    j.th = std::thread([jp, file, t, iter, N, E, ndof, composite, el_part, el_local, el_N, el_offset]() {
      if (cudaEventSynchronize(jp->done) != cudaSuccess) { jp->err = "state copy failed"; return; }
      const double* Q = jp->pinned[0];
      if (composite) {
        jp->order.resize(size_t(ndof));
        for (int e = 0; e < E; ++e) {
          const size_t n = size_t(el_N[e] + 1) * (el_N[e] + 1) * 4;
          std::memcpy(jp->order.data() + el_offset[e], jp->pinned[el_part[e]] + size_t(el_local[e]) * n,
                      n * sizeof(double));
        }
        Q = jp->order.data();
      }
      if (hg_write_restart(file.c_str(), t, iter, Q, ndof, N, E) != 0) jp->err = hg_restart_last_error();
    });
    return 0;
  } catch (const std::exception& ex) { return fail_ctx(c, ex.what()); }
}

extern "C" int hg_restart_wait(hg_ctx* c) {
  if (!c) return 1;
  autosave_finish(c);
  if (c->autosave && !c->autosave->err.empty()) return fail_ctx(c, "restart write: " + c->autosave->err);
  return 0;
}
