// Context, errors, scratch arena and DPD size math of libcpsd_b200.
#include "runtime.hpp"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>

namespace cpsd {

const i64 ZORB[8] = {1, 0, 0, 0, 0, 0, 0, 0};

static thread_local std::string g_err;

int set_error(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

const std::string &last_error() { return g_err; }

int cuda_check(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return CPSD_OK;
    return set_error(CPSD_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

Context &ctx() {
    thread_local Context c;
    return c;
}

// irpdso (src/libsrint/irpdso.f:1-52)
i64 irpdso(i64 sym, const i64 *popp, const i64 *popq, i64 iop) {
    i64 n = 0;
    for (i64 r = 1; r <= ctx().nirrep; r++) {
        i64 l = dp(r, sym);
        if (iop == 1) {
            n += popp[l - 1] * popq[r - 1];
        } else if (iop == 0 || iop == 2) {
            if (l > r) continue;
            if (l < r) n += popp[l - 1] * popq[r - 1];
            else if (iop == 0) n += popp[l - 1] * (popq[r - 1] - 1) / 2;
            else n += popp[l - 1] * (popq[r - 1] + 1) / 2;
        }
    }
    return n;
}

// idsymsoc (src/libsrint/idsymsoc.f:1-30)
i64 idsymsoc(i64 irrepx, const i64 *popp, const i64 *popq, i64 ioppq, const i64 *popr,
             const i64 *pops, i64 ioprs) {
    i64 n = 0;
    for (i64 r = 1; r <= ctx().nirrep; r++) n += irpdso(dp(r, irrepx), popp, popq, ioppq) * irpdso(r, popr, pops, ioprs);
    return n;
}

// isymoffso (src/libsrint/isymoffso.f:1-54)
i64 isymoffso(i64 irrepq1, i64 irrep, const i64 *popp, const i64 *popq, i64 iop) {
    i64 off = 1;
    for (i64 q = 1; q <= irrepq1 - 1; q++) {
        i64 p = dp(q, irrep);
        if (iop == 1) off += popp[p - 1] * popq[q - 1];
        else if (p < q) off += popp[p - 1] * popq[q - 1];
        else if (p == q) off += popp[p - 1] * (popp[q - 1] + (iop == 2 ? 1 : -1)) / 2;
    }
    return off;
}

i64 Desc::block_base(i64 R) const {
    i64 b = 0;
    for (i64 r = 1; r < R; r++) b += nleft(dp(r, sym)) * nright(r);
    return b;
}

std::string Desc::key() const {
    std::string s;
    char buf[32];
    for (int k = 0; k < 4; k++)
        for (int i = 0; i < 8; i++) {
            snprintf(buf, sizeof buf, "%lld,", (long long)pop[k][i]);
            s += buf;
        }
    snprintf(buf, sizeof buf, "|%lld%lld|%lld", (long long)iop[0], (long long)iop[1], (long long)sym);
    return s + buf;
}

Desc make_desc(const i64 *p0, const i64 *p1, const i64 *p2, const i64 *p3, i64 iop0, i64 iop1, i64 sym) {
    Desc d;
    memcpy(d.pop[0], p0, sizeof d.pop[0]);
    memcpy(d.pop[1], p1, sizeof d.pop[0]);
    memcpy(d.pop[2], p2, sizeof d.pop[0]);
    memcpy(d.pop[3], p3, sizeof d.pop[0]);
    d.iop[0] = iop0;
    d.iop[1] = iop1;
    d.sym = sym;
    return d;
}

Desc desc_of(const cpsd_opt *t) {
    return make_desc(t->popp, t->popq, t->popr, t->pops, t->ioppq, t->ioprs, t->sym);
}

std::mutex &upload_mutex() {
    static std::mutex m;
    return m;
}

bool mem_trace_on() {
    static const bool on = getenv("CPSD_TRACE_MEM") != nullptr;
    return on;
}

double host_ms() {
    static const auto t0 = std::chrono::steady_clock::now();
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void mem_trace(const char *what, size_t bytes, double ms, bool ok) {
    if (!mem_trace_on()) return;
    fprintf(stderr, "[cpsd mem] t=%.1f ms %s %.3f GB%s (%.2f ms)\n", host_ms(), what, bytes / 1e9, ok ? "" : " FAILED",
            ms);
}

// ------------------------------------------------------------------ arena
Arena &arena() {
    thread_local Arena a;
    return a;
}

void Arena::set_external(void *p, size_t bytes) {
    free_all();
    external = true;
    chunks.push_back({(char *)p, bytes, false});
}

void Arena::free_all() {
    for (auto &c : chunks)
        if (c.owned) cudaFree(c.base);
    chunks.clear();
    cur_chunk = cur_off = in_use = 0;
    external = false;
}

void Arena::trim() {
    while (chunks.size() > cur_chunk + 1 && chunks.back().owned) {
        const double t = mem_trace_on() ? host_ms() : 0.0;
        cudaFree(chunks.back().base);
        if (mem_trace_on()) mem_trace("arena trim cudaFree", chunks.back().size, host_ms() - t);
        chunks.pop_back();
    }
}

int Arena::alloc(size_t bytes, void **out) {
    bytes = (bytes + 255) & ~(size_t)255;
    while (cur_chunk < chunks.size()) {
        Chunk &c = chunks[cur_chunk];
        if (cur_off + bytes <= c.size) {
            *out = c.base + cur_off;
            cur_off += bytes;
            in_use += bytes;
            if (in_use > high_water) high_water = in_use;
            return CPSD_OK;
        }
        if (cur_chunk + 1 >= chunks.size()) break;
        cur_chunk++;
        cur_off = 0;
    }
    if (external)
        return set_error(CPSD_EMEM, "workspace too small: need " + std::to_string(bytes) + " more bytes");
    // room for what follows: up to 1 GiB beyond the request (256 MiB at least)
    size_t sz = bytes + std::min(bytes, (size_t)1 << 30);
    if (sz < ((size_t)256 << 20)) sz = (size_t)256 << 20;
    void *p = nullptr;
    const double t0 = mem_trace_on() ? host_ms() : 0.0;
    const bool first_ok = cudaMalloc(&p, sz) == cudaSuccess;
    if (mem_trace_on()) mem_trace("arena cudaMalloc", sz, host_ms() - t0, first_ok);
    if (!first_ok) {
        cudaGetLastError();
        sz = bytes;
        if (cudaMalloc(&p, sz) != cudaSuccess) {
            cudaGetLastError();
            // an idle pool buffer of up to twice the size (plus 1 GiB)
            // becomes the chunk (no driver call: at the memory limit a
            // cudaFree would wait for the whole device), else the idle cached
            // copies of earlier runs give way
            size_t got = 0;
            p = pool_take_idle(sz, 2 * sz + ((size_t)1 << 30), &got);
            if (p) {
                sz = got;
                mem_trace("arena chunk from an idle pool buffer", sz, 0.0);
            } else {
                pool_release_idle();
            }
            if (!p && cudaMalloc(&p, sz) != cudaSuccess) {
                cudaGetLastError();
                // then the copies this run keeps for later operations
                if (!evict_cached_copies(sz) || cudaMalloc(&p, sz) != cudaSuccess) {
                    cudaGetLastError();
                    return set_error(CPSD_EMEM,
                                     "cudaMalloc of scratch failed (" + std::to_string(bytes) + " bytes)");
                }
            }
        }
    }
    chunks.push_back({(char *)p, sz, true});
    cur_chunk = chunks.size() - 1;
    cur_off = bytes;
    *out = p;
    in_use += bytes;
    if (in_use > high_water) high_water = in_use;
    return CPSD_OK;
}

}  // namespace cpsd
