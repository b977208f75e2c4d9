// Serving loop: assembly requests on resident templates, admitted against
// the HBM budget onto execution slots (one stream each) by a server thread,
// so that requests that arrive while others run overlap on the device.
//
// A request runs the value path of slgpu_matrix_process on the template's
// resident groups and pattern -- coefficients (with the request's
// per-element data gathered into each group's element order), contraction,
// CSR values -- on its slot's stream, then copies the values to the host.
// The pattern, meshes, tables and addresses are never rebuilt.
#include "engine_internal.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <thread>

namespace slgpu {

static void cuda_check_srv(cudaError_t e, const char* what)
{
    if (e != cudaSuccess)
        throw SlgpuException(SLGPU_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// dst[r][e] = src[r][elems[e]]: per-element data from mesh order into the
// group's element order.
__global__ void k_gather_elements(const double* __restrict__ src, const int32_t* __restrict__ elems, int64_t nelem, int rows,
                                  int64_t count, double* __restrict__ dst)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nelem * rows)
        return;
    const int64_t r = i / nelem, e = i - r * nelem;
    dst[i] = src[r * count + elems[e]];
}

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t ticket = 0;
    int handle = 0, precision = 0;
    struct Update {
        int group, kind, index, rows;
        int64_t count;
        int64_t offset;  // in doubles, within the request's input block
    };
    std::vector<Update> updates;
    double* in = nullptr;  // page-locked block with every update's values
    size_t in_cap = 0;
    int64_t nin = 0;
    // Caller arrays already page-locked: read in place (host pointer, offset
    // in doubles, count), no copy at submit.
    struct DirectIn {
        const double* host;
        int64_t offset, n;
    };
    std::vector<DirectIn> direct_in;
    // Template requests (slgpu_server_submit_template): process the matrix
    // once (pattern build and first values) with these constraint flags.
    bool is_template = false;
    std::vector<uint8_t> constr;
    // SLGPU_UPDATE_SCALES: group and its term scales then multipliers.
    std::vector<std::pair<int, std::vector<double>>> scales;
    std::vector<DevBuf> ts;  // device term scales while running
    double* Aout = nullptr;
    double* Dout = nullptr;
    bool pinned_out = false;
    // Template state kept alive while the request runs.
    std::shared_ptr<Matrix> tmpl;
    int64_t est_bytes = 0;
    // Device and host resources while running.
    DevBuf vals, Avals, Dvals, upd;
    std::vector<DevBuf> ed, fd;
    int64_t nnzA = 0, nnzD = 0;
    int status = -1;  // -1 queued, -2 running, else the final status
    std::string error;
    double t_submit = 0, t_start = 0, t_done = 0, dev_ms = 0, launch_ms = 0;
    double parts_ms[3] = {0, 0, 0};
    int slot = -1;
};

struct Slot {
    Exec ex;
    size_t arena_need = 0;  // largest arena use (fitted or missed) of a request so far
    cudaEvent_t start = nullptr, done = nullptr;
    std::shared_ptr<Request> req;
    void* pinned = nullptr;  // staging for inputs and pageable outputs
    size_t pinned_bytes = 0;
    unsigned int* err_host = nullptr;  // page-locked copy of the split-precision error flag
};

}  // namespace

struct Server {
    Ctx* ctx = nullptr;
    std::vector<Slot> slots;
    std::thread th;
    std::mutex mu;  // queue, request table, stop flag
    std::condition_variable wake, done_cv;
    std::deque<std::shared_ptr<Request>> queue;
    std::map<int64_t, std::shared_ptr<Request>> reqs;
    int64_t next_ticket = 1;
    int64_t running = 0;
    bool stop = false;
    Clock::time_point t0 = Clock::now();
    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
    // Page-locked blocks for request inputs, reused by size class (under mu).
    std::multimap<size_t, void*> pin_free;
    std::vector<void*> pin_all;
};

namespace {

// Device bytes a request allocates while it runs (r == nullptr: a request
// that updates every per-element array of every group).
int64_t estimate_bytes(const Matrix& M, int precision, const Request* r)
{
    int64_t vals = 0, coef = 0, exps = 0, split = 0;
    for (auto& g : M.groups) {
        vals += (int64_t)g->ntf * g->ndof * g->nelem;
        coef += (int64_t)g->nterms * g->ngp * g->nelem;
        exps += g->nelem;
        // The split groups of a request are sliced and contracted together:
        // their column slices coexist.
        const int64_t Qpad = ((int64_t)g->nterms * g->ngp + 31) / 32 * 32;
        split += 7 * Qpad * (int64_t)g->tiles.size() * 64 + (int64_t)g->tiles.size() * 256 + 512;
    }
    for (auto& f : M.frags) vals += (int64_t)f->nr * f->nc;
    int64_t upd = 0, over = 0;
    if (r != nullptr) {
        upd = r->nin;
        for (auto& u : r->updates) {
            const GroupDev& g = *M.groups[u.group];
            over += (u.kind == SLGPU_UPDATE_ELEMDATA ? (int64_t)g.elemdata.bytes() : (int64_t)g.fielddata.bytes()) / 8;
        }
    } else {
        for (auto& g : M.groups) over += (int64_t)(g->elemdata.bytes() + g->fielddata.bytes()) / 8;
        upd = over;
    }
    const int64_t csr = M.pattern ? M.pattern->nnzA + M.pattern->nnzD : 0;
    int64_t b = 8 * (vals + coef + csr + upd + over) + 4 * exps;
    if (precision != SLGPU_PREC_FP64)
        b += split;
    return b + (int64_t(1) << 20);
}

void ensure_pinned(Slot& s, size_t bytes)
{
    if (s.pinned_bytes >= bytes)
        return;
    if (s.pinned != nullptr)
        cudaFreeHost(s.pinned);
    s.pinned = nullptr;
    s.pinned_bytes = 0;
    cuda_check_srv(cudaHostAlloc(&s.pinned, bytes, cudaHostAllocDefault), "cudaHostAlloc");
    s.pinned_bytes = bytes;
}

// Issues a request on its slot (server thread, context lock held).
void launch(Server& S, Slot& s, Request& r)
{
    Ctx* ctx = S.ctx;
    const Matrix& M = *r.tmpl;
    Pattern& P = *M.pattern;
    const double t0 = S.now();
    ctx->x = &s.ex;
    stage_reset(s.ex);
    htrace_begin(ctx);
    cudaStream_t st = s.ex.stream;
    // Request buffers come from the slot's arena, grown (rarely, on this
    // slot's stream) to the largest request seen.
    {
        const size_t want = std::max<size_t>(s.arena_need, (size_t)r.est_bytes);
        if (s.ex.arena.bytes() < want)
            s.ex.arena.alloc(ctx, want + want / 8);
        s.ex.arena_off = 0;
        s.ex.arena_miss = 0;
        s.ex.arena_on = true;
    }
    htrace_mark(ctx, "request: arena");
    cuda_check_srv(cudaEventRecord(s.start, st), "cudaEventRecord");
    // Inputs: every update's values are in the request's page-locked block
    // (filled at submit): one copy to the device, then per updated group a
    // copy of its resident array (unless the update replaces all of it) with
    // the slice replaced by the gathered values.
    r.nnzA = P.nnzA;
    r.nnzD = P.nnzD;
    const size_t outbytes = r.pinned_out ? 0 : (size_t)(r.nnzA + r.nnzD) * 8;
    if (outbytes > 0)
        ensure_pinned(s, outbytes + 64);
    std::vector<GroupData> ov(M.groups.size());
    r.ed.clear();
    r.fd.clear();
    r.ed.resize(M.groups.size());
    r.fd.resize(M.groups.size());
    if (r.nin > 0) {
        r.upd.alloc(ctx, (size_t)r.nin * 8);
        if (!r.direct_in.empty()) {
            for (const auto& d : r.direct_in)
                cuda_check_srv(cudaMemcpyAsync(r.upd.as<double>() + d.offset, d.host, (size_t)d.n * 8, cudaMemcpyHostToDevice, st),
                               "H2D request inputs");
        } else {
            cuda_check_srv(cudaMemcpyAsync(r.upd.as<void>(), r.in, (size_t)r.nin * 8, cudaMemcpyHostToDevice, st),
                           "H2D request inputs");
        }
        for (auto& u : r.updates) {
            GroupDev& g = *M.groups[u.group];
            const bool elem = u.kind == SLGPU_UPDATE_ELEMDATA;
            DevBuf& dst = elem ? r.ed[u.group] : r.fd[u.group];
            const DevBuf& res = elem ? g.elemdata : g.fielddata;
            const bool whole = elem ? g.elemdata_off.size() == 1 : g.field_off.size() == 1;
            if (dst.empty()) {
                dst.alloc(ctx, res.bytes());
                if (!whole)
                    cuda_check_srv(cudaMemcpyAsync(dst.as<void>(), res.as<void>(), res.bytes(), cudaMemcpyDeviceToDevice, st),
                                   "D2D group data");
            }
            const int64_t base = elem ? g.elemdata_off[u.index] : g.field_off[u.index];
            const int64_t n = g.nelem * u.rows;
            if (n > 0) {
                k_gather_elements<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(r.upd.as<double>() + u.offset, g.elems.as<int32_t>(),
                                                                            g.nelem, u.rows, u.count, dst.as<double>() + base);
                cuda_check_srv(cudaGetLastError(), "k_gather_elements");
                ctx->launches++;
            }
            (elem ? ov[u.group].elemdata : ov[u.group].fielddata) = dst.as<double>();
        }
    }
    r.ts.clear();
    r.ts.resize(r.scales.size());
    for (size_t k = 0; k < r.scales.size(); k++) {
        const int gi = r.scales[k].first;
        upload_staged(ctx, r.ts[k], r.scales[k].second.data(), (size_t)M.groups[gi]->nterms * 8);
        ov[gi].term_scale = r.ts[k].as<double>();
    }
    const double t1 = S.now();
    htrace_mark(ctx, "request: inputs");
    std::vector<int64_t> gvb;
    int64_t total_vals = 0;
    // Element values stored as process() stores them (floats for FP32-level
    // requests whose groups all go through the split kernels).
    const bool f32v = float_values(M, r.precision);
    std::vector<Segment> segs = build_segments(M, &gvb, &total_vals, f32v);
    r.vals.alloc(ctx, (size_t)std::max<int64_t>(total_vals, 1) * 8);
    ctx->x->kev_tag.clear();
    launch_contractions(ctx, M, r.precision, gvb, r.vals.as<double>(), &ov, f32v);
    const double t2 = S.now();
    r.Avals.alloc(ctx, (size_t)std::max<int64_t>(P.nnzA, 1) * 8);
    r.Dvals.alloc(ctx, (size_t)std::max<int64_t>(P.nnzD, 1) * 8);
    std::vector<RowSeg> rsegs = row_segments(M, segs, f32v);
    // Destination multipliers of the request's scale updates (segments are
    // the groups' destinations in order).
    if (!r.scales.empty()) {
        std::vector<size_t> sbase(M.groups.size() + 1, 0);
        for (size_t gi = 0; gi < M.groups.size(); gi++) sbase[gi + 1] = sbase[gi] + M.groups[gi]->ndests;
        for (const auto& sc : r.scales) {
            const GroupDev& g = *M.groups[sc.first];
            for (int d = 0; d < g.ndests; d++) rsegs[sbase[sc.first] + d].mult = sc.second[g.nterms + d];
        }
    }
    DevBuf dsegs;
    upload_staged(ctx, dsegs, rsegs.data(), rsegs.size() * sizeof(RowSeg));
    launch_row_values(ctx, M, P, rsegs, dsegs.as<RowSeg>(), false, r.vals.as<double>(), r.Avals.as<double>(), r.Dvals.as<double>());
    r.vals.release();  // stream-ordered: after the value kernel
    double* hA = r.pinned_out ? r.Aout : static_cast<double*>(s.pinned);
    double* hD = r.pinned_out ? r.Dout : static_cast<double*>(s.pinned) + r.nnzA;
    if (r.nnzA > 0)
        cuda_check_srv(cudaMemcpyAsync(hA, r.Avals.as<void>(), (size_t)r.nnzA * 8, cudaMemcpyDeviceToHost, st), "D2H Avals");
    if (r.nnzD > 0 && hD != nullptr)
        cuda_check_srv(cudaMemcpyAsync(hD, r.Dvals.as<void>(), (size_t)r.nnzD * 8, cudaMemcpyDeviceToHost, st), "D2H Dvals");
    *s.err_host = 0;
    if (r.precision != SLGPU_PREC_FP64 && !s.ex.split_error.empty())
        cuda_check_srv(cudaMemcpyAsync(s.err_host, s.ex.split_error.as<void>(), 4, cudaMemcpyDeviceToHost, st), "D2H split error");
    cuda_check_srv(cudaEventRecord(s.done, st), "cudaEventRecord");
    htrace_mark(ctx, "request: outputs");
    s.ex.arena_on = false;
    s.arena_need = std::max(s.arena_need, s.ex.arena_off + s.ex.arena_miss);
    ctx->x = &ctx->main;
    const double t3 = S.now();
    r.parts_ms[0] = (t1 - t0) * 1e3;
    r.parts_ms[1] = (t2 - t1) * 1e3;
    r.parts_ms[2] = (t3 - t2) * 1e3;
}

// Completion of the request on slot s (server thread, context lock held).
void finish(Server& S, Slot& s)
{
    Request& r = *s.req;
    Ctx* ctx = S.ctx;
    int status = SLGPU_OK;
    std::string msg;
    cudaError_t e = cudaEventQuery(s.done);
    if (e != cudaSuccess) {
        status = SLGPU_E_CUDA;
        msg = std::string("request failed on the device: ") + cudaGetErrorString(e);
    } else {
        float ms = 0;
        cudaEventElapsedTime(&ms, s.start, s.done);
        r.dev_ms = ms;
        if (*s.err_host != 0) {
            status = SLGPU_E_TIMEOUT;
            msg = "a split-precision contraction tile timed out waiting for its data";
        }
        if (!r.pinned_out) {
            const double* hp = static_cast<const double*>(s.pinned);
            if (r.nnzA > 0)
                std::memcpy(r.Aout, hp, (size_t)r.nnzA * 8);
            if (r.nnzD > 0 && r.Dout != nullptr)
                std::memcpy(r.Dout, hp + r.nnzA, (size_t)r.nnzD * 8);
        }
    }
    // Device buffers: freed in the slot stream's order (its work is done).
    ctx->x = &s.ex;
    r.Avals.release();
    r.Dvals.release();
    r.upd.release();
    r.ed.clear();
    r.fd.clear();
    r.ts.clear();
    r.tmpl.reset();
    ctx->x = &ctx->main;
    std::lock_guard<std::mutex> lk(S.mu);
    if (r.in != nullptr) {
        S.pin_free.emplace(r.in_cap, r.in);
        r.in = nullptr;
    }
    r.t_done = S.now();
    r.status = status;
    r.error = msg;
    S.running--;
    s.req.reset();
    S.done_cv.notify_all();
}

void server_loop(Server& S)
{
    Ctx* ctx = S.ctx;
    cudaSetDevice(ctx->device);
    for (;;) {
        bool progress = false;
        // Completions.
        for (Slot& s : S.slots) {
            if (!s.req)
                continue;
            if (cudaEventQuery(s.done) == cudaErrorNotReady)
                continue;
            std::lock_guard<std::recursive_mutex> cl(ctx->mu);
            finish(S, s);
            progress = true;
        }
        // Admissions, in arrival order.
        for (;;) {
            Slot* free_slot = nullptr;
            for (Slot& s : S.slots)
                if (!s.req) {
                    free_slot = &s;
                    break;
                }
            std::shared_ptr<Request> r;
            {
                std::lock_guard<std::mutex> lk(S.mu);
                if (free_slot == nullptr || S.queue.empty())
                    break;
                r = S.queue.front();
            }
            std::lock_guard<std::recursive_mutex> cl(ctx->mu);
            // Device memory the request adds: what its slot's arena lacks.
            const int64_t extra = std::max<int64_t>(0, r->est_bytes - (int64_t)free_slot->ex.arena.bytes());
            if (ctx->in_use + extra > (int64_t)ctx->budget) {
                bool busy = false;
                for (Slot& s : S.slots) busy = busy || (bool)s.req;
                if (busy)
                    break;  // wait for memory to free up
            }
            {
                std::lock_guard<std::mutex> lk(S.mu);
                S.queue.pop_front();
                r->t_start = S.now();
                r->status = -2;
                r->slot = (int)(free_slot - S.slots.data());
            }
            if (r->is_template) {
                // A new template: its pattern build synchronises the main
                // stream (the slots' streams keep running); it completes here.
                const double tl = S.now();
                slgpu_csr_info info{};
                const int code = slgpu_matrix_process(reinterpret_cast<slgpu_ctx*>(ctx), r->handle, r->constr.data(), r->precision, &info);
                std::lock_guard<std::mutex> lk(S.mu);
                r->launch_ms = (S.now() - tl) * 1e3;
                r->status = code;
                if (code != SLGPU_OK)
                    r->error = ctx->last_error;
                r->t_done = S.now();
                r->slot = -1;
                S.running--;
                S.done_cv.notify_all();
                progress = true;
                continue;
            }
            free_slot->req = r;
            int code = SLGPU_OK;
            std::string msg;
            try {
                const double tl = S.now();
                launch(S, *free_slot, *r);
                r->launch_ms = (S.now() - tl) * 1e3;
            } catch (const SlgpuException& e) {
                code = e.e.code;
                msg = e.e.msg;
            } catch (const std::exception& e) {
                code = SLGPU_E_ARG;
                msg = e.what();
            }
            if (code != SLGPU_OK) {
                free_slot->ex.arena_on = false;
                ctx->x = &ctx->main;
                cudaStreamSynchronize(free_slot->ex.stream);
                std::lock_guard<std::mutex> lk(S.mu);
                r->status = code;
                r->error = msg;
                if (r->in != nullptr) {
                    S.pin_free.emplace(r->in_cap, r->in);
                    r->in = nullptr;
                }
                r->t_done = S.now();
                r->Avals.release();
                r->Dvals.release();
                r->vals.release();
                r->upd.release();
                r->ed.clear();
                r->fd.clear();
                r->tmpl.reset();
                S.running--;
                free_slot->req.reset();
                S.done_cv.notify_all();
            }
            progress = true;
        }
        std::unique_lock<std::mutex> lk(S.mu);
        bool busy = false;
        for (Slot& s : S.slots) busy = busy || (bool)s.req;
        if (S.stop && S.queue.empty() && !busy)
            break;
        if (!progress) {
            if (busy)
                S.wake.wait_for(lk, std::chrono::microseconds(20));
            else
                S.wake.wait_for(lk, std::chrono::milliseconds(5));
        }
    }
}

}  // namespace
}  // namespace slgpu

using namespace slgpu;

struct slgpu_server : public slgpu::Server {};
struct slgpu_ctx : public slgpu::Ctx {};

extern "C" {

int slgpu_server_create(slgpu_ctx* ctx, int nslots, slgpu_server** out)
{
    if (ctx == nullptr || out == nullptr || nslots < 1 || nslots > 64)
        return SLGPU_E_ARG;
    *out = nullptr;
    if (ctx->record_only) {
        ctx->last_error = "no CUDA device: a record-only context cannot serve requests";
        return SLGPU_E_NODEVICE;
    }
    std::lock_guard<std::recursive_mutex> cl(ctx->mu);
    cudaSetDevice(ctx->device);
    auto* S = new slgpu_server();
    S->ctx = ctx;
    S->slots.resize(nslots);
    for (Slot& s : S->slots) {
        if (cudaStreamCreateWithFlags(&s.ex.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&s.start) != cudaSuccess || cudaEventCreate(&s.done) != cudaSuccess) {
            ctx->last_error = "cannot create the server's streams";
            slgpu_server_destroy(S);
            return SLGPU_E_CUDA;
        }
        for (auto& e : s.ex.ev) cudaEventCreate(&e);
        if (cudaHostAlloc(reinterpret_cast<void**>(&s.err_host), 16, cudaHostAllocDefault) != cudaSuccess) {
            ctx->last_error = "cannot allocate page-locked memory";
            slgpu_server_destroy(S);
            return SLGPU_E_CUDA;
        }
        *s.err_host = 0;
    }
    S->th = std::thread([S] { server_loop(*S); });
    *out = S;
    return SLGPU_OK;
}

int slgpu_server_submit(slgpu_server* S, const slgpu_request* rq, int64_t* ticket)
{
    if (S == nullptr || rq == nullptr || ticket == nullptr)
        return SLGPU_E_ARG;
    Ctx* ctx = S->ctx;
    auto r = std::make_shared<Request>();
    std::map<std::pair<const double*, int64_t>, int64_t> seen_arrays;  // (values, doubles) -> offset
    {
        std::lock_guard<std::recursive_mutex> cl(ctx->mu);
        auto it = ctx->matrices.find(rq->handle);
        if (it == ctx->matrices.end()) {
            ctx->last_error = "unknown matrix handle " + std::to_string(rq->handle);
            return SLGPU_E_ARG;
        }
        Matrix& M = *it->second;
        if (!M.pattern) {
            ctx->last_error = "a template must be processed once before it serves requests";
            return SLGPU_E_ARG;
        }
        if (rq->precision != SLGPU_PREC_FP64 && rq->precision != SLGPU_PREC_SPLIT && rq->precision != SLGPU_PREC_FP32) {
            ctx->last_error = "unknown precision mode";
            return SLGPU_E_ARG;
        }
        if (rq->Avals == nullptr || (M.pattern->nnzD > 0 && rq->Dvals == nullptr)) {
            ctx->last_error = "request output buffers missing";
            return SLGPU_E_ARG;
        }
        // The request keeps the template's resident parts alive, not its
        // value buffers (a shallow copy of the matrix description).
        auto t = std::make_shared<Matrix>();
        t->ndofs = M.ndofs;
        t->groups = M.groups;
        t->frags = M.frags;
        t->pattern = M.pattern;
        r->tmpl = t;
        auto& seen = seen_arrays;  // identical arrays are sent once
        for (int i = 0; i < rq->nupdates; i++) {
            const slgpu_update& u = rq->updates[i];
            if (u.group < 0 || u.group >= (int)M.groups.size()) {
                ctx->last_error = "update: group index out of range";
                return SLGPU_E_ARG;
            }
            const GroupDev& g = *M.groups[u.group];
            if (u.kind == SLGPU_UPDATE_SCALES) {
                if (u.rows != g.nterms + g.ndests || u.count != 1 || u.values == nullptr) {
                    ctx->last_error = "update: scales need rows = nterms + ndests, count = 1";
                    return SLGPU_E_ARG;
                }
                std::vector<double> v(u.values, u.values + u.rows);
                if (group_symmetric(g))
                    for (int t = 0; t < g.nterms; t++)
                        if (std::memcmp(&v[t], &v[g.mirror[t]], sizeof(double)) != 0) {
                            ctx->last_error = "update: the scales break the symmetry of a symmetric group (mirror terms differ)";
                            return SLGPU_E_ARG;
                        }
                r->scales.emplace_back(u.group, std::move(v));
                continue;
            }
            const bool elem = u.kind == SLGPU_UPDATE_ELEMDATA;
            if (!elem && u.kind != SLGPU_UPDATE_FIELDDATA) {
                ctx->last_error = "update: unknown kind";
                return SLGPU_E_ARG;
            }
            const int narr = elem ? (int)g.elemdata_off.size() : (int)g.field_off.size();
            if (u.index < 0 || u.index >= narr) {
                ctx->last_error = "update: array index out of range";
                return SLGPU_E_ARG;
            }
            const int rows = elem ? 1 : g.field_rows[u.index];
            if (u.rows != rows) {
                ctx->last_error = "update: row count does not match the array";
                return SLGPU_E_ARG;
            }
            const auto& types = ctx->meshes.at(g.mesh).types;
            const int64_t mesh_n = types.count(g.elemtype) ? types.at(g.elemtype).nelem : 0;
            if (u.count != mesh_n || u.values == nullptr) {
                ctx->last_error = "update: count must be the number of mesh elements of the group's type";
                return SLGPU_E_ARG;
            }
            const int64_t n = (int64_t)rows * u.count;
            auto it = seen.find({u.values, n});
            int64_t off = r->nin;
            if (it == seen.end()) {
                seen[{u.values, n}] = off;
                r->nin += n;
            } else
                off = it->second;
            r->updates.push_back(Request::Update{u.group, u.kind, u.index, rows, u.count, off});
        }
        r->handle = rq->handle;
        r->precision = rq->precision;
        r->Aout = rq->Avals;
        r->Dout = rq->Dvals;
        cudaPointerAttributes pa{}, pd{};
        const bool pA = cudaPointerGetAttributes(&pa, rq->Avals) == cudaSuccess && pa.type == cudaMemoryTypeHost;
        const bool pD = rq->Dvals == nullptr ||
                        (cudaPointerGetAttributes(&pd, rq->Dvals) == cudaSuccess && pd.type == cudaMemoryTypeHost);
        cudaGetLastError();
        r->pinned_out = pA && pD;
        r->est_bytes = estimate_bytes(M, rq->precision, r.get());
        if (r->est_bytes > (int64_t)ctx->budget) {
            ctx->last_error = "a request needs more device memory than the whole HBM budget";
            return SLGPU_E_BUDGET;
        }
    }
    // Inputs: page-locked caller arrays are read in place by the request's
    // copy; others are copied into a page-locked block here (outside the
    // context lock), so that the caller may reuse them at once.
    if (r->nin > 0) {
        bool pinned = true;
        for (const auto& kv : seen_arrays) {
            cudaPointerAttributes a{};
            pinned = pinned && cudaPointerGetAttributes(&a, kv.first.first) == cudaSuccess && a.type == cudaMemoryTypeHost;
        }
        cudaGetLastError();
        if (pinned)
            for (const auto& kv : seen_arrays) r->direct_in.push_back(Request::DirectIn{kv.first.first, kv.second, kv.first.second});
    }
    if (r->nin > 0 && r->direct_in.empty()) {
        const size_t need = (size_t)r->nin * 8;
        size_t cap = size_t(1) << 16;
        while (cap < need) cap <<= 1;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            auto it = S->pin_free.lower_bound(cap);
            if (it != S->pin_free.end() && it->first == cap) {
                r->in = static_cast<double*>(it->second);
                S->pin_free.erase(it);
            }
        }
        if (r->in == nullptr) {
            void* p = nullptr;
            if (cudaHostAlloc(&p, cap, cudaHostAllocDefault) != cudaSuccess) {
                cudaGetLastError();
                ctx->last_error = "cannot allocate page-locked memory for the request inputs";
                return SLGPU_E_BUDGET;
            }
            r->in = static_cast<double*>(p);
            std::lock_guard<std::mutex> lk(S->mu);
            S->pin_all.push_back(p);
        }
        r->in_cap = cap;
        // Every distinct data array once, at its offset ((values, doubles) -> offset).
        for (const auto& kv : seen_arrays) std::memcpy(r->in + kv.second, kv.first.first, (size_t)kv.first.second * 8);
    }
    std::lock_guard<std::mutex> lk(S->mu);
    r->ticket = S->next_ticket++;
    r->t_submit = S->now();
    S->reqs[r->ticket] = r;
    S->queue.push_back(r);
    S->running++;
    *ticket = r->ticket;
    S->wake.notify_one();
    return SLGPU_OK;
}

int slgpu_server_submit_template(slgpu_server* S, int handle, const uint8_t* isconstrained, int precision, int64_t* ticket)
{
    if (S == nullptr || ticket == nullptr)
        return SLGPU_E_ARG;
    Ctx* ctx = S->ctx;
    auto r = std::make_shared<Request>();
    {
        std::lock_guard<std::recursive_mutex> cl(ctx->mu);
        auto it = ctx->matrices.find(handle);
        if (it == ctx->matrices.end()) {
            ctx->last_error = "unknown matrix handle " + std::to_string(handle);
            return SLGPU_E_ARG;
        }
        const Matrix& M = *it->second;
        if (precision != SLGPU_PREC_FP64 && precision != SLGPU_PREC_SPLIT && precision != SLGPU_PREC_FP32) {
            ctx->last_error = "unknown precision mode";
            return SLGPU_E_ARG;
        }
        r->is_template = true;
        r->handle = handle;
        r->precision = precision;
        r->constr.assign((size_t)M.ndofs + 1, 0);
        if (isconstrained != nullptr)
            std::memcpy(r->constr.data(), isconstrained, (size_t)M.ndofs);
        // The pattern build's device memory: sort keys and indices, runs,
        // slot map and incidences of every COO entry, values and CSR arrays.
        int64_t ncoo = 0, nvals = 0;
        for (auto& g : M.groups) {
            ncoo += (int64_t)g->ntf * g->ndof * g->nelem * g->ndests;
            nvals += (int64_t)g->ntf * g->ndof * g->nelem;
        }
        for (auto& f : M.frags) {
            ncoo += (int64_t)f->nr * f->nc;
            nvals += (int64_t)f->nr * f->nc;
        }
        r->est_bytes = 40 * ncoo + 24 * nvals + 16 * M.ndofs + (int64_t(1) << 20);
        if (r->est_bytes > (int64_t)ctx->budget) {
            ctx->last_error = "the template's first assembly needs more device memory than the whole HBM budget";
            return SLGPU_E_BUDGET;
        }
    }
    std::lock_guard<std::mutex> lk(S->mu);
    r->ticket = S->next_ticket++;
    r->t_submit = S->now();
    S->reqs[r->ticket] = r;
    S->queue.push_back(r);
    S->running++;
    *ticket = r->ticket;
    S->wake.notify_one();
    return SLGPU_OK;
}

int slgpu_server_wait(slgpu_server* S, int64_t ticket, double timeout_s, slgpu_request_stats* stats)
{
    if (S == nullptr)
        return SLGPU_E_ARG;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end())
        return SLGPU_E_ARG;
    std::shared_ptr<Request> r = it->second;
    auto done = [&] { return r->status >= 0; };
    if (timeout_s < 0)
        S->done_cv.wait(lk, done);
    else
        S->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
    if (stats != nullptr) {
        stats->submit_s = r->t_submit;
        stats->start_s = r->t_start;
        stats->done_s = r->t_done;
        stats->device_ms = r->dev_ms;
        stats->slot = r->slot;
        stats->status = r->status;
        stats->launch_ms = r->launch_ms;
        for (int i = 0; i < 3; i++) stats->launch_parts_ms[i] = r->parts_ms[i];
    }
    if (!done())
        return SLGPU_E_TIMEOUT;
    return r->status;
}

int slgpu_server_error(slgpu_server* S, int64_t ticket, char* buf, size_t len)
{
    if (S == nullptr || buf == nullptr || len == 0)
        return SLGPU_E_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end())
        return SLGPU_E_ARG;
    std::snprintf(buf, len, "%s", it->second->error.c_str());
    return SLGPU_OK;
}

int slgpu_server_release(slgpu_server* S, int64_t ticket)
{
    if (S == nullptr)
        return SLGPU_E_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end() || it->second->status < 0)
        return SLGPU_E_ARG;
    S->reqs.erase(it);
    return SLGPU_OK;
}

int64_t slgpu_server_pending(slgpu_server* S)
{
    if (S == nullptr)
        return 0;
    std::lock_guard<std::mutex> lk(S->mu);
    return S->running;
}

double slgpu_server_clock(slgpu_server* S) { return S == nullptr ? 0.0 : S->now(); }

int slgpu_server_prepare(slgpu_server* S, int handle, int precision)
{
    if (S == nullptr)
        return SLGPU_E_ARG;
    Ctx* ctx = S->ctx;
    std::lock_guard<std::recursive_mutex> cl(ctx->mu);
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->running > 0) {
            ctx->last_error = "a server is prepared while it has no requests";
            return SLGPU_E_ARG;
        }
    }
    auto it = ctx->matrices.find(handle);
    if (it == ctx->matrices.end() || !it->second->pattern) {
        ctx->last_error = "prepare: unknown or unprocessed template " + std::to_string(handle);
        return SLGPU_E_ARG;
    }
    if (precision != SLGPU_PREC_FP64 && precision != SLGPU_PREC_SPLIT && precision != SLGPU_PREC_FP32) {
        ctx->last_error = "unknown precision mode";
        return SLGPU_E_ARG;
    }
    const Matrix& M = *it->second;
    try {
        cudaSetDevice(ctx->device);
        const size_t est = (size_t)estimate_bytes(M, precision, nullptr);
        for (Slot& s : S->slots) {
            ctx->x = &s.ex;
            prepare_value_path(ctx, M, precision);
            const size_t want = std::max(s.arena_need, est);
            if (s.ex.arena.bytes() < want)
                s.ex.arena.alloc(ctx, want + want / 8);
            s.arena_need = want;
            ctx->x = &ctx->main;
        }
        for (Slot& s : S->slots) cuda_check_srv(cudaStreamSynchronize(s.ex.stream), "prepare");
    } catch (const SlgpuException& e) {
        ctx->x = &ctx->main;
        ctx->last_error = e.e.msg;
        return e.e.code;
    }
    return SLGPU_OK;
}

void slgpu_server_destroy(slgpu_server* S)
{
    if (S == nullptr)
        return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->wake.notify_all();
    }
    if (S->th.joinable())
        S->th.join();
    Ctx* ctx = S->ctx;
    std::lock_guard<std::recursive_mutex> cl(ctx->mu);
    cudaSetDevice(ctx->device);
    for (Slot& s : S->slots) {
        if (s.ex.stream != nullptr)
            cudaStreamSynchronize(s.ex.stream);
        // Slot buffers go before their stream.
        s.ex.split_cols.release();
        s.ex.split_colexp.release();
        s.ex.split_error.release();
        s.ex.arena.release();
        if (s.ex.stream != nullptr)
            cudaStreamSynchronize(s.ex.stream);
        for (auto& e : s.ex.ev)
            if (e != nullptr)
                cudaEventDestroy(e);
        for (auto& e : s.ex.evpool) cudaEventDestroy(e);
        for (auto& e : s.ex.kev) cudaEventDestroy(e);
        if (s.start != nullptr)
            cudaEventDestroy(s.start);
        if (s.done != nullptr)
            cudaEventDestroy(s.done);
        if (s.pinned != nullptr)
            cudaFreeHost(s.pinned);
        if (s.err_host != nullptr)
            cudaFreeHost(s.err_host);
        stage_free(s.ex);
        if (s.ex.stream != nullptr)
            cudaStreamDestroy(s.ex.stream);
    }
    for (void* p : S->pin_all) cudaFreeHost(p);
    delete S;
}

int slgpu_host_alloc(slgpu_ctx* ctx, size_t bytes, void** out)
{
    if (ctx == nullptr || out == nullptr)
        return SLGPU_E_ARG;
    *out = nullptr;
    if (ctx->record_only)
        return SLGPU_E_NODEVICE;
    cudaSetDevice(ctx->device);
    if (cudaHostAlloc(out, std::max<size_t>(bytes, 16), cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return SLGPU_E_BUDGET;
    }
    return SLGPU_OK;
}

void slgpu_host_free(void* p)
{
    if (p != nullptr)
        cudaFreeHost(p);
}

}  // extern "C"
