// kmm_hoststate.cu -- time steps with the state held in host arrays.
//
// The reference keeps its prognostic fields in host arrays and its time loop calls the solver
// routines on them every step (main_dns.f90:198-811).  kmm_bind_host names the host array of a
// field; kmm_run_host then runs steps the way such a loop would with an accelerator in its place:
// before every step each bound field is copied from its host array to the device, and after every
// step it is copied back, so the host arrays hold each step's result.
//
// The copies run on two streams of their own, one per direction, in pieces of at most
// HS_CHUNK bytes.  After a step, its downloads (device -> host) and the next step's uploads
// (host -> device) proceed together: each chunk's upload waits only for the download of the same
// chunk, so the two copy engines work at once and the next step waits for the last upload only.
// The history fields' downloads (fn^{n-1} and the like, whose new value is the buffer the step
// takes over from fn) start before the step and run during it.
#include <new>
#include <vector>

#include "kmm_internal.cuh"

// bytes per copy: a whole field up to 64 MB.  Smaller pieces shorten the wait of the first upload
// behind its download but cost more per copy; at 128 x 129 x 128 (17 MB fields) 4 MB pieces made a
// step's copies 8 % slower than whole fields
#define HS_CHUNK ((size_t)64 << 20)

namespace {

struct HostBind {
    int field;
    void *host;
    size_t bytes;
};

struct Chunk {
    int bind;        // index into KmmHostState::binds
    size_t off, n;   // byte range of the field
};

struct KmmHostState {
    std::vector<HostBind> binds;
    std::vector<Chunk> chunks;
    std::vector<const void *> early_src;   // per binding: the buffer its early download read (or NULL)
    std::vector<cudaEvent_t> down_ev;   // one per chunk: its download has finished
    cudaStream_t h2d = NULL, d2h = NULL;
    cudaEvent_t entry_ev = NULL, up_ev = NULL, step_ev = NULL;
};

KmmHostState *hs_of(kmm_ctx *ctx) { return reinterpret_cast<KmmHostState *>(ctx->hoststate); }

// fields whose host layout is the device layout (the 3/2-grid physical fields and imatrix go
// through a layout transform in kmm_upload / kmm_download and cannot be bound)
bool bindable(int f) {
    return (f >= 0 && f < KMM_NSPECTRAL) || (f >= KMM_U0 && f < KMM_NMEAN_END) ||
           (f >= KMM_BCTOP && f < KMM_NWALL_END) || (f >= KMM_XPART && f < KMM_NPART_END);
}

int hs_streams(kmm_ctx *ctx, KmmHostState *S) {
    if (!S->h2d) CK(cudaStreamCreateWithFlags(&S->h2d, cudaStreamNonBlocking));
    if (!S->d2h) CK(cudaStreamCreateWithFlags(&S->d2h, cudaStreamNonBlocking));
    if (!S->entry_ev) CK(cudaEventCreateWithFlags(&S->entry_ev, cudaEventDisableTiming));
    if (!S->up_ev) CK(cudaEventCreateWithFlags(&S->up_ev, cudaEventDisableTiming));
    if (!S->step_ev) CK(cudaEventCreateWithFlags(&S->step_ev, cudaEventDisableTiming));
    // the chunk list and its events follow the bindings
    S->chunks.clear();
    for (size_t b = 0; b < S->binds.size(); ++b)
        for (size_t off = 0; off < S->binds[b].bytes; off += HS_CHUNK) {
            const size_t n = S->binds[b].bytes - off < HS_CHUNK ? S->binds[b].bytes - off : HS_CHUNK;
            S->chunks.push_back(Chunk{(int)b, off, n});
        }
    while (S->down_ev.size() < S->chunks.size()) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        S->down_ev.push_back(e);
    }
    return KMM_OK;
}

// device address of a chunk: the field's current buffer (the history exchanges of a step move the
// buffers between fields, so it is looked up when the copy is enqueued)
char *chunk_dev(kmm_ctx *ctx, const KmmHostState *S, const Chunk &c) {
    char *d = (char *)kmm_field_ptr(ctx, S->binds[c.bind].field);
    return d ? d + c.off : NULL;
}

// a chunk whose download ran during the step (its field took over the buffer that download read)
bool downloaded_early(kmm_ctx *ctx, const KmmHostState *S, const Chunk &c) {
    return c.bind < (int)S->early_src.size() && S->early_src[c.bind] &&
           kmm_field_ptr(ctx, S->binds[c.bind].field) == S->early_src[c.bind];
}

// every bound field host -> device on h2d; the chunk waits for its own download when `after_down`,
// and the chunks downloaded during the step go first (their downloads have finished or will soon)
int enqueue_uploads(kmm_ctx *ctx, KmmHostState *S, bool after_down) {
    for (int pass = after_down ? 0 : 1; pass < 2; ++pass)
        for (size_t i = 0; i < S->chunks.size(); ++i) {
            const Chunk &c = S->chunks[i];
            if (after_down && downloaded_early(ctx, S, c) != (pass == 0)) continue;
            char *d = chunk_dev(ctx, S, c);
            if (!d) return KMM_ERR_NOMEM;
            if (after_down) CK(cudaStreamWaitEvent(S->h2d, S->down_ev[i], 0));
            CK(cudaMemcpyAsync(d, (const char *)S->binds[c.bind].host + c.off, c.n, cudaMemcpyHostToDevice, S->h2d));
        }
    CK(cudaEventRecord(S->up_ev, S->h2d));
    CK(cudaStreamWaitEvent(ctx->stream, S->up_ev, 0));   // the step reads what has landed
    return KMM_OK;
}

// the n field whose buffer a history field n-1 takes over in a step (the step exchanges the two
// buffers and writes only the new n: fn^{n-1} = fn^n, main_dns.f90:268-275, 335, 386, 418), or -1
int hist_partner(int f) {
    if (f == KMM_FNM1) return KMM_FN;
    if (f == KMM_GNM1) return KMM_GN;
    if (f == KMM_SCNM1) return KMM_SCN;
    if (f >= KMM_C11NM1 && f <= KMM_C33NM1) return KMM_C11N + (f - KMM_C11NM1);
    if (f >= KMM_STR11NM1 && f <= KMM_STR33NM1) return KMM_STR11N + (f - KMM_STR11NM1);
    return -1;
}

// before a step: the bound history fields' results are the n fields' current buffers, which the
// step reads but does not write, so their downloads start now and run during the step (after this
// step's uploads have read the host arrays)
int enqueue_early_downloads(kmm_ctx *ctx, KmmHostState *S) {
    S->early_src.assign(S->binds.size(), NULL);
    bool any = false;
    for (size_t i = 0; i < S->chunks.size(); ++i) {
        const Chunk &c = S->chunks[i];
        const int n = hist_partner(S->binds[c.bind].field);
        if (n < 0) continue;
        const char *d = (const char *)kmm_field_ptr(ctx, n);
        if (!d) return KMM_ERR_NOMEM;
        if (!any) CK(cudaStreamWaitEvent(S->d2h, S->up_ev, 0));
        any = true;
        S->early_src[c.bind] = d;
        CK(cudaMemcpyAsync((char *)S->binds[c.bind].host + c.off, d + c.off, c.n, cudaMemcpyDeviceToHost, S->d2h));
        CK(cudaEventRecord(S->down_ev[i], S->d2h));
    }
    return KMM_OK;
}

// every bound field device -> host on d2h, after the work enqueued so far on the context's stream;
// a history field downloaded early is skipped if the step made that buffer its own (else, e.g. when
// the step stopped before its exchanges, it is downloaded again here)
int enqueue_downloads(kmm_ctx *ctx, KmmHostState *S) {
    CK(cudaEventRecord(S->step_ev, ctx->stream));
    CK(cudaStreamWaitEvent(S->d2h, S->step_ev, 0));
    for (size_t i = 0; i < S->chunks.size(); ++i) {
        const Chunk &c = S->chunks[i];
        if (downloaded_early(ctx, S, c)) continue;
        const char *d = chunk_dev(ctx, S, c);
        if (!d) return KMM_ERR_NOMEM;
        CK(cudaMemcpyAsync((char *)S->binds[c.bind].host + c.off, d, c.n, cudaMemcpyDeviceToHost, S->d2h));
        CK(cudaEventRecord(S->down_ev[i], S->d2h));
    }
    return KMM_OK;
}

}  // namespace

void kmm_hoststate_release(kmm_ctx *ctx) {
    KmmHostState *S = hs_of(ctx);
    if (!S) return;
    if (S->d2h) cudaStreamSynchronize(S->d2h);
    if (S->h2d) cudaStreamSynchronize(S->h2d);
    for (cudaEvent_t e : S->down_ev) cudaEventDestroy(e);
    if (S->entry_ev) cudaEventDestroy(S->entry_ev);
    if (S->up_ev) cudaEventDestroy(S->up_ev);
    if (S->step_ev) cudaEventDestroy(S->step_ev);
    if (S->h2d) cudaStreamDestroy(S->h2d);
    if (S->d2h) cudaStreamDestroy(S->d2h);
    delete S;
    ctx->hoststate = NULL;
}

extern "C" int kmm_bind_host(kmm_ctx *ctx, int field, void *host, size_t bytes) {
    if (!ctx) return KMM_ERR_ARG;
    if (field < 0 && !host) {   // clear every binding
        if (ctx->hoststate) hs_of(ctx)->binds.clear();
        return KMM_OK;
    }
    size_t n;
    int b;
    if (!bindable(field) || kmm_field_info(ctx, field, &n, &b)) {
        kmm_set_error(ctx, "kmm_bind_host: field %d cannot be bound (spectral, mean-mode, wall and particle fields can)",
                      field);
        return KMM_ERR_ARG;
    }
    if (host && bytes != n * (size_t)b) {
        kmm_set_error(ctx, "kmm_bind_host: field %d expects %zu bytes, got %zu", field, n * (size_t)b, bytes);
        return KMM_ERR_ARG;
    }
    if (!ctx->hoststate) ctx->hoststate = new (std::nothrow) KmmHostState();
    KmmHostState *S = hs_of(ctx);
    if (!S) return KMM_ERR_NOMEM;
    for (size_t i = 0; i < S->binds.size(); ++i)
        if (S->binds[i].field == field) {
            S->binds.erase(S->binds.begin() + i);
            break;
        }
    if (host && bytes) S->binds.push_back(HostBind{field, host, bytes});
    return KMM_OK;
}

extern "C" int kmm_run_host(kmm_ctx *ctx, int n) {
    if (!ctx || n < 0) return KMM_ERR_ARG;
    KmmHostState *S = hs_of(ctx);
    if (!S || S->binds.empty()) return kmm_run(ctx, n);
    RET(hs_streams(ctx, S));
    if (n == 0) return KMM_OK;
    // the first uploads follow whatever the context's stream holds
    CK(cudaEventRecord(S->entry_ev, ctx->stream));
    CK(cudaStreamWaitEvent(S->h2d, S->entry_ev, 0));
    RET(enqueue_uploads(ctx, S, false));
    int st = KMM_OK;
    for (int s = 0; s < n; ++s) {
        st = enqueue_early_downloads(ctx, S);
        if (st) break;
        st = kmm_step(ctx);
        if (st == KMM_ERR_CUDA || st == KMM_ERR_NOMEM || st == KMM_ERR_ARG) break;
        // the host arrays receive this step's result even when the step reports a stop status
        const int dst = enqueue_downloads(ctx, S);
        if (dst) { st = dst; break; }
        if (st != KMM_OK) break;
        if (s + 1 < n) {
            const int ust = enqueue_uploads(ctx, S, true);
            if (ust) { st = ust; break; }
        }
    }
    if (S->d2h) {
        const cudaError_t e1 = cudaStreamSynchronize(S->d2h), e2 = cudaStreamSynchronize(S->h2d);
        if ((e1 != cudaSuccess || e2 != cudaSuccess) && st == KMM_OK) {
            kmm_set_error(ctx, "kmm_run_host: copy failed: %s",
                          cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
            st = KMM_ERR_CUDA;
        }
    }
    return st;
}
