// runtime.cu -- device selection, stream, status word and error policy shared
// by the gpunb_* / gpupot_ / irr_simd_* entry points of libnb6b200.
//
// Device choice mirrors GPUNB_devinit (gpunb.velocity.cu:575-627): the
// GPU_LIST environment variable (space-separated ids) is honoured, first id
// wins since this library drives one GPU per process; NB_GPU_DEVICE is an
// explicit override; otherwise device (irank % device_count), as the
// single-GPU build does (gpunb.gpu.cu:574).
//
// Error policy: the reference asserts and aborts on bad input (NAN_CHECK,
// ni range, gpunb.velocity.cu:40,751,802).  This library does the same by
// default.  nb6_set_abort_on_error_(0) switches to "record and return": the
// call does no work and nb6_last_status_() reports the code.
#include "nb6_common.cuh"
#include "copy_pool.h"

#include <string.h>

static int g_device = -1;
static int g_num_sms = 0;
static cudaStream_t g_stream = nullptr;
static int *g_dev_status = nullptr;
static int *g_status_host = nullptr;   // pinned copy, filled by nb6_status_fetch
static bool g_status_fetched = false;
static bool g_uva = false;
static int g_host_status = 0;
static int g_abort_on_error = 1;
static bool g_abort_env_read = false;

static void read_abort_env() {
    if (g_abort_env_read) return;
    g_abort_env_read = true;
    const char *e = getenv("NB6_ABORT_ON_ERROR");
    if (e) g_abort_on_error = atoi(e) != 0;
}

void nb6_set_host_status(int code) {
    if (g_host_status == 0) g_host_status = code;
}

void nb6_fatal(int code) {
    read_abort_env();
    nb6_set_host_status(code);
    if (g_abort_on_error) {
        fprintf(stderr, "libnb6b200: fatal error code %d, aborting\n", code);
        abort();
    }
}

void nb6_devinit_once(int irank) {
    if (g_device >= 0) return;
    read_abort_env();
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        fprintf(stderr, "libnb6b200: no CUDA device visible\n");
        nb6_fatal(NB6_ERR_CUDA);
        return;
    }
    int dev = (irank >= 0 ? irank : 0) % count;
    if (const char *gl = getenv("GPU_LIST")) {
        char buf[256];
        strncpy(buf, gl, sizeof(buf) - 1);
        buf[sizeof(buf) - 1] = 0;
        char *p = strtok(buf, " ,");
        if (p) dev = atoi(p) % count;
    }
    if (const char *nd = getenv("NB_GPU_DEVICE")) dev = atoi(nd) % count;
    g_device = dev;
    NB6_CUDA_CHECK(cudaSetDevice(dev));
    NB6_CUDA_CHECK(cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev));
    NB6_CUDA_CHECK(cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking));
    NB6_CUDA_CHECK(cudaMalloc((void **)&g_dev_status, sizeof(int)));
    NB6_CUDA_CHECK(cudaMemset(g_dev_status, 0, sizeof(int)));
    NB6_CUDA_CHECK(cudaMallocHost((void **)&g_status_host, sizeof(int)));
    *g_status_host = 0;
    int uva = 0;
    NB6_CUDA_CHECK(cudaDeviceGetAttribute(&uva, cudaDevAttrUnifiedAddressing, dev));
    g_uva = uva != 0;
    if (getenv("NB6_VERBOSE")) {
        cudaDeviceProp prop;
        cudaGetDeviceProperties(&prop, dev);
        fprintf(stderr, "# libnb6b200 GPU initialization - rank: %d; device: %d %s; SMs %d\n",
                irank, dev, prop.name, g_num_sms);
    }
}

int nb6_device_id() { return g_device; }
static CopyPool g_pool;
static int g_open_libs = 0;

CopyPool &nb6_copy_pool() {
    g_pool.start(CopyPool::default_parts());
    return g_pool;
}
void nb6_lib_opened() { ++g_open_libs; }
void nb6_lib_closed() {
    if (--g_open_libs <= 0) {
        g_open_libs = 0;
        g_pool.stop();
    }
}

int nb6_num_sms() { return g_num_sms; }
cudaStream_t nb6_stream() { return g_stream; }
int *nb6_dev_status() { return g_dev_status; }

bool nb6_uva() { return g_uva; }

// Enqueue a copy of the device status word into pinned host memory; the
// next nb6_check_dev_status after a sync of `st` reads that copy instead of
// doing a synchronous copy of its own.
void nb6_status_fetch(cudaStream_t st) {
    NB6_CUDA_CHECK(cudaMemcpyAsync(g_status_host, g_dev_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    g_status_fetched = true;
}

// Read (and clear) the device status word; call after a stream sync.
int nb6_check_dev_status() {
    int st = 0;
    if (g_status_fetched) {
        st = *(volatile int *)g_status_host;
        g_status_fetched = false;
    } else {
        NB6_CUDA_CHECK(cudaMemcpy(&st, g_dev_status, sizeof(int), cudaMemcpyDeviceToHost));
    }
    if (st != 0) {
        NB6_CUDA_CHECK(cudaMemset(g_dev_status, 0, sizeof(int)));
        fprintf(stderr, "libnb6b200: device reported status %d\n", st);
        nb6_fatal(st);
    }
    return st;
}

extern "C" {

// Extension entry points (no reference counterpart): error policy + status.
void nb6_set_abort_on_error_(int *flag) {
    g_abort_env_read = true;
    g_abort_on_error = (*flag != 0);
}

int nb6_last_status_() {
    int s = g_host_status;
    g_host_status = 0;
    return s;
}

int nb6_device_() { return g_device; }

}  // extern "C"
