// status.cu -- status codes, last-error bookkeeping, device buffers, mode.
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <mutex>
#include <string>

#include "common.cuh"

namespace mdbas {

thread_local long long *g_launch_counter = nullptr;

namespace {
std::atomic<int> g_last_status{MDBAS_NB_OK};
std::mutex g_msg_mutex;
std::string g_last_msg;
int g_mode = -1;
}  // namespace

void set_last_status(int st, const char *msg) {
  g_last_status.store(st);
  if (msg) {
    std::lock_guard<std::mutex> lk(g_msg_mutex);
    g_last_msg = msg;
  }
}

int cuda_fail(cudaError_t err, const char *what, const char *file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s failed at %s:%d: %s", what, file, line, cudaGetErrorString(err));
  set_last_status(MDBAS_NB_ERR_CUDA, buf);
  if (err == cudaErrorMemoryAllocation) return MDBAS_NB_ERR_ALLOC;
  if (err == cudaErrorNoDevice || err == cudaErrorInsufficientDriver) return MDBAS_NB_ERR_NO_DEVICE;
  return MDBAS_NB_ERR_CUDA;
}

int DBuf::ensure(size_t n) {
  if (n == 0) n = 16;
  if (n <= bytes) return MDBAS_NB_OK;
  release();
  cudaError_t e = cudaMalloc(&p, n);
  if (e != cudaSuccess) {
    p = nullptr;
    cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
    return MDBAS_NB_ERR_ALLOC;
  }
  bytes = n;
  return MDBAS_NB_OK;
}

void DBuf::release() {
  if (p) cudaFree(p);  // errors during process teardown are ignored
  p = nullptr;
  bytes = 0;
}

const char *last_message() {
  static thread_local std::string copy;
  std::lock_guard<std::mutex> lk(g_msg_mutex);
  copy = g_last_msg;
  return copy.c_str();
}

}  // namespace mdbas

extern "C" {

const char *mdbas_nb_status_string(int status) {
  switch (status) {
    case MDBAS_NB_OK: return "ok";
    case MDBAS_NB_ERR_ARG: return "invalid argument";
    case MDBAS_NB_ERR_CUDA: return "CUDA runtime error";
    case MDBAS_NB_ERR_NO_DEVICE: return "no usable CUDA device";
    case MDBAS_NB_ERR_ALLOC: return "allocation failed";
    case MDBAS_NB_ERR_CAPACITY: return "list capacity exceeded";
    case MDBAS_NB_ERR_BOX: return "box too small or atom outside the box";
    case MDBAS_NB_ERR_LINKCELL: return "too few link cells for the link ratio";
    case MDBAS_NB_ERR_EXCL: return "invalid exclusion topology";
    case MDBAS_NB_ERR_UNSUPPORTED: return "option not supported on this path";
    case MDBAS_NB_ERR_OVERFLOW: return "fixed-point accumulator overflow";
    case MDBAS_NB_ERR_NONFINITE: return "non-finite coordinates";
    case MDBAS_NB_ERR_MISSING: return "a MDBas routine this call delegates to is not linked";
    case MDBAS_NB_ERR_STATE: return "call out of order";
    default: return "unknown status";
  }
}

int mdbas_nb_last_status(void) { return mdbas::g_last_status.load(); }

const char *mdbas_nb_last_message(void) { return mdbas::last_message(); }

int mdbas_nb_version(void) { return 100; }

int mdbas_nb_build_arch(void) { return 1000; }

int mdbas_nb_get_mode(void) {
  if (mdbas::g_mode < 0) {
    const char *m = getenv("MDBAS_NB_MODE");
    mdbas::g_mode = (m && (strcmp(m, "mixed") == 0 || strcmp(m, "1") == 0)) ? 1 : 0;
  }
  return mdbas::g_mode;
}

int mdbas_nb_set_mode(int mode) {
  if (mode != 0 && mode != 1) return MDBAS_NB_ERR_ARG;
  mdbas::g_mode = mode;
  return MDBAS_NB_OK;
}

}  // extern "C"
