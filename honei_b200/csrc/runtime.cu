// Runtime pieces of the B200 backend: error reporting, per-stream device
// workspaces for the fused reductions, launch accounting.
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>

namespace hb2
{
    static thread_local std::string t_last_error;
    static thread_local uint64_t t_launches = 0;
    int g_num_sms = 0;

    void set_error(const std::string & msg) { t_last_error = msg; }

    int fail(int status, const std::string & msg)
    {
        set_error(msg);
        return status;
    }

    int cuda_status(cudaError_t e, const char * where)
    {
        set_error(std::string(where) + ": " + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? HB2_ERR_NOMEM : HB2_ERR_CUDA;
    }

    // off by default: inside CUDA graphs on B200 the launch gaps are already
    // hidden (measured: MG level 10 3.349 ms with, 3.343 ms without; level 11
    // 6.73 / 6.51 ms); HB2_PDL=1 turns it on
    int64_t l2_prefetch_rows(size_t)
    {
        const char * v = getenv("HB2_Q1_PREFETCH");
        const double w = v && *v ? atof(v) : 0.0;
        return w > 0 ? (int64_t)(w * num_sms() * 2048.0) : 0;
    }

    bool pdl_enabled()
    {
        static const bool on = getenv("HB2_PDL") && strcmp(getenv("HB2_PDL"), "1") == 0;
        return on;
    }

    void count_launches(uint64_t n) { t_launches += n; }
    void set_launch_count(uint64_t n) { t_launches = n; }

    int num_sms()
    {
        if (g_num_sms == 0)
        {
            int dev = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
            if (g_num_sms <= 0) g_num_sms = 148;
        }
        return g_num_sms;
    }

    int workspace_create(Workspace ** out, uint32_t max_blocks)
    {
        Workspace * w = new Workspace();
        w->max_blocks = max_blocks;
        cudaGetDevice(&w->device);
        // one allocation: partials | group partials | scalars | tickets | barrier words, error flag
        const uint32_t max_tickets = 1u << 16;
        const uint32_t ngpart = max_blocks / kReduceGroup + 4096;
        size_t bytes = sizeof(double) * (max_blocks + ngpart + 64) + sizeof(unsigned) * max_tickets + 64;
        char * base = 0;
        cudaError_t e = cudaMalloc(&base, bytes);
        if (e != cudaSuccess) { delete w; return cuda_status(e, "workspace cudaMalloc"); }
        e = cudaMemset(base, 0, bytes);
        if (e != cudaSuccess) { cudaFree(base); delete w; return cuda_status(e, "workspace cudaMemset"); }
        w->partials = (double *)base;
        w->gpart = w->partials + max_blocks;
        w->scalars = w->gpart + ngpart;
        unsigned * words = (unsigned *)(w->scalars + 64);
        w->ticket = words;
        w->max_tickets = max_tickets;
        w->bar_words = words + max_tickets;
        w->error = (int *)(words + max_tickets + 4);
        e = cudaMallocHost(&w->host_scalars, sizeof(double) * 64);
        if (e != cudaSuccess) { cudaFree(base); delete w; return cuda_status(e, "workspace cudaMallocHost"); }
        *out = w;
        return HB2_OK;
    }

    void workspace_destroy(Workspace * w)
    {
        if (! w) return;
        cudaFree(w->partials);
        cudaFreeHost(w->host_scalars);
        delete w;
    }

    // Fused reductions on one stream share a ticket counter, so each
    // (device, stream) pair gets its own workspace; kernels of one stream
    // never overlap, kernels of different streams never share a counter.
    static std::mutex g_ws_mutex;
    static std::map<std::pair<int, cudaStream_t>, Workspace *> g_ws;

    int stream_workspace(cudaStream_t stream, Workspace ** out)
    {
        int dev = 0;
        HB2_CUDA(cudaGetDevice(&dev));
        std::lock_guard<std::mutex> lock(g_ws_mutex);
        std::pair<int, cudaStream_t> key(dev, stream);
        std::map<std::pair<int, cudaStream_t>, Workspace *>::iterator it = g_ws.find(key);
        if (it != g_ws.end()) { *out = it->second; return HB2_OK; }
        Workspace * w = 0;
        int st = workspace_create(&w, kMaxReduceBlocks);
        if (st != HB2_OK) return st;
        g_ws[key] = w;
        *out = w;
        return HB2_OK;
    }

    int default_workspace(Workspace ** out) { return stream_workspace(0, out); }
}

extern "C" const char * hb2_last_error(void) { return hb2::t_last_error.c_str(); }

extern "C" const char * hb2_version(void) { return "honei_b200 0.1 (sm_100a)"; }

extern "C" uint64_t hb2_launch_count(void) { return hb2::t_launches; }

extern "C" uint64_t hb2_workspace_count(void)
{
    std::lock_guard<std::mutex> lock(hb2::g_ws_mutex);
    return hb2::g_ws.size();
}
