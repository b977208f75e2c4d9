// Internal declarations of the slgpu assembly engine (not part of the C ABI).
#pragma once

#include "slgpu.h"

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <exception>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace slgpu {

struct Ctx;

// Device allocation owned by a context; counts against its HBM budget.
class DevBuf {
public:
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept { *this = std::move(o); }
    DevBuf& operator=(DevBuf&& o) noexcept;
    ~DevBuf() { release(); }
    void alloc(Ctx* ctx, size_t bytes);  // throws on failure / budget
    void release();
    template <class T> T* as() const { return static_cast<T*>(p_); }
    size_t bytes() const { return n_; }
    bool empty() const { return p_ == nullptr; }

private:
    Ctx* ctx_ = nullptr;
    cudaStream_t s_ = nullptr;  // allocated (and freed) in this stream's order
    void* p_ = nullptr;
    size_t n_ = 0;
    bool arena_ = false;  // carved from an execution state's arena (nothing to free)
};

struct Error {
    int code;
    std::string msg;
};

struct SlgpuException : std::exception {
    Error e;
    SlgpuException(int code, std::string msg) : e{code, std::move(msg)} {}
    const char* what() const noexcept override { return e.msg.c_str(); }
};

// One instruction of a compiled coefficient program (register-allocated DAG).
struct Instr {
    int32_t op, dst, a, b;
};
enum { INSTR_STORE = 100 };
constexpr int kMaxSlots = 48;

// Orientation-uniform run of elements processed by one contraction tile row.
struct Tile {
    int32_t e0, ne, orient, pad;
};

struct MeshDev {
    int64_t nnodes = 0;
    DevBuf xyz;
    std::vector<double> hxyz;  // record-only copy
    struct Type {
        int ncn = 0;
        int64_t nelem = 0;
        DevBuf conn;
        std::vector<int32_t> hconn;  // record-only copy
    };
    std::map<int, Type> types;
};

// A group after upload: everything a launch needs, plus host-side metadata.
struct GroupDev {
    int mesh = 0, elemtype = 0, elemdim = 0, problemdim = 0;
    int64_t nelem = 0;
    int norient = 1, ngp = 0, ncn = 0, ntf = 0, ndof = 0, nterms = 0, ndests = 0;
    bool rhs = false;
    std::vector<Instr> prog;
    std::vector<int64_t> tab_off;
    std::vector<int32_t> tab_rows;
    std::vector<int64_t> elemdata_off;
    std::vector<int64_t> field_off;
    std::vector<int32_t> field_rows;
    std::vector<double> term_scale;
    std::vector<int32_t> term_tf, term_dof;
    std::vector<double> dest_mult;
    std::vector<Tile> tiles;
    uint64_t addr_hash[2] = {0, 0};
    // Coefficient program as given (for the runtime-compiled kernel) and a
    // hash of the geometry inputs (groups with equal hashes share J, detJ).
    std::vector<slgpu_node> nodes;
    std::vector<int> term_node;
    std::vector<double> hconsts;
    uint64_t geom_hash = 0;
    uint64_t serial = 0;  // unique per group created by the context
    // Runtime-compiled coefficient kernel of the batch this group leads
    // (batch members by serial).
    mutable std::vector<uint64_t> jit_members;
    mutable cudaKernel_t jit_kernel = nullptr;

    DevBuf elems, orient, weights, lagrange, tables, consts, prog_d, elemdata, fielddata, field_off_d, field_rows_d,
        tab_off_d, tab_rows_d, term_scale_d, term_tf_d, term_dof_d, tiles_d;
    std::vector<std::shared_ptr<DevBuf>> tfaddr, dofaddr;  // per destination; shared by groups of one matrix when allowed

    // Mirror of each term for symmetric element matrices (empty: none), and
    // whether mirror coefficients are equal bit for bit; see mirror_terms in
    // engine.cu.
    std::vector<int32_t> mirror;
    bool mirror_exact = false;
    // Content keys for transposed pairs of groups (cross_pairs in engine.cu):
    // per term its test-function table, dof table and coefficient expression
    // (up to the order of factors), and per element / field data array its
    // values (updated when an array is replaced).
    struct Key {
        uint64_t a = 0, b = 0;
        bool operator==(const Key& o) const { return a == o.a && b == o.b; }
    };
    struct TermKey {
        Key tf, dof, coef;
    };
    std::vector<TermKey> term_keys;
    std::vector<Key> data_keys;  // elemdata arrays, then fielddata arrays

    // Split-precision operand A (row slices of M), built on first use per
    // tier (0 split, 1 FP32 level) and form (0 every entry; 1 the upper
    // triangle of a symmetric group and 2 every entry of a group with a
    // transposed partner, each row mapped to an entry and its mirror):
    // slot tier + 2 form.
    struct Split {
        int S = 0, L = 0, Qpad = 0, Ppad = 0, nrows = 0;
        DevBuf slices, rowexp, rowmap;
    };
    std::unique_ptr<Split> split[6];
    // FP64 tensor-core operand M^T per form (0 every entry, 1 upper triangle
    // of a symmetric group, 2 every entry with its transposed partner's).
    struct Fp64Mt {
        int Qpad = 0, rpad = 0, nrows = 0;
        DevBuf Mt, rowmap;
    };
    std::unique_ptr<Fp64Mt> fmt[3];

    // Record-only copy of the original description (for inspection).
    struct Record;
    std::shared_ptr<Record> rec;
};

struct FragmentDev {
    int32_t ntr = 0, ndr = 0, nr = 0;
    int64_t nc = 0;
    DevBuf rows, cols, vals;
    uint64_t addr_hash[2] = {0, 0};
    std::vector<int32_t> hrows, hcols;  // record-only copies
    std::vector<double> hvals;
};

// Resident COO -> CSR mapping (pattern), reusable while addresses and
// constraints are unchanged.  The numeric phase only needs the CSR structure,
// the per-row incidence lists and the slot map.
struct Pattern {
    uint64_t key[2] = {0, 0};
    uint64_t serial = 0;   // unique per pattern built by the context
    int64_t ndofs = 0, nA = 0, nD = 0, nnzA = 0, nnzD = 0, ncoo = 0, nvalid = 0, ninc = 0;
    int lmax = 0;          // longest row (A and D entries)
    int row_kernel = -1;   // CSR value kernel chosen by timing: 0 streaming warps, 1 warp per row, -1 not yet
    DevBuf Arows, Acols, Drows, Dcols;
    DevBuf ainds, dinds;   // int32 [nA], [nD]: global DOF of each local row of A / column of D
    DevBuf slotmap;        // int16 [ncoo]: position in the row's [A | D] segment, -1 = dropped
    DevBuf inc_ptr;        // uint32 [nA+1]: incidences of each row
    DevBuf inc;            // uint64 [ninc]: segment << 40 | COO index of the incidence's first entry
    uint64_t last_use = 0;
    // Right-hand-side patterns: the rows (DOFs) that receive at least one
    // entry, ascending, on the host and the device (built on first use).
    bool rhs_rows_ready = false;
    std::vector<int32_t> rhs_rows;
    DevBuf rhs_rows_d;
};

// Per COO segment, as the CSR value kernels read it: where its entries
// values start in the element-value buffer, its destination multiplier, the
// width of its incidences (ndof of a group, 1 for a raw fragment) and whether
// the values are stored as floats (FP32-level steps, float_values(): entry k
// of the segment is float number 2 * val_base + k of the buffer).
struct RowSeg {
    int64_t coo_base;
    int64_t val_base;
    double mult;
    int32_t width, f32;
};

struct Segment {
    int64_t coo_base;
    int64_t count;
    int64_t val_base;
    double mult;
};

// The value path of one matrix's process() on a resident pattern
// (coefficients, contractions, CSR values) captured as one CUDA graph.  It is
// replayed while `sig` -- every device pointer and host value that the
// captured launches bake in -- is unchanged.
struct ValueGraph {
    std::vector<uint64_t> sig;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<char*> stage;  // page-locked blocks read by the graph's copies
    std::vector<std::pair<std::string, double>> kev_tag;  // kernel-family timers recorded by the graph
    int64_t launches = 0;                                 // kernels per replay
    std::shared_ptr<Pattern> pattern;                     // kept resident while the graph exists
    ValueGraph() = default;
    ValueGraph(const ValueGraph&) = delete;
    ValueGraph& operator=(const ValueGraph&) = delete;
    ~ValueGraph();
};

struct Matrix {
    int64_t ndofs = 0;
    std::vector<std::shared_ptr<GroupDev>> groups;
    std::vector<std::shared_ptr<FragmentDev>> frags;
    std::shared_ptr<Pattern> pattern;
    DevBuf vals;  // contraction outputs + fragment values
    DevBuf Avals, Dvals;
    std::vector<uint8_t> rec_constrained;  // record-only
    slgpu_csr_info info{};
    // Graph of the value path, and the signature of the last ungraphed run
    // (a graph is captured when two consecutive runs have equal signatures).
    std::unique_ptr<ValueGraph> vgraph;
    std::vector<uint64_t> vsig_prev;
    bool graph_failed = false;  // capture was refused: this matrix runs ungraphed
    // Segments of the value kernels, resident (replayed graphs read them);
    // updated in place when multipliers change.
    std::vector<RowSeg> rsegs_host;
    DevBuf rsegs_dev;
    // slgpu_matrix_share_addresses: the device copies and content hashes of
    // the address arrays given to add_group since the last process(), by host
    // pointer and length.
    struct SharedAddresses {
        std::shared_ptr<DevBuf> buf;
        uint64_t hash[2];
    };
    bool share_addresses = false;
    std::map<std::pair<const void*, int64_t>, SharedAddresses> shared_addresses;
};

// Per kernel family: device time (CUDA events around each launch on the
// stream), launches and algorithmic work of the last process().
struct KernelStat {
    double ms = 0, work = 0;
    int64_t launches = 0;
};

// Everything a sequence of launches needs for itself: its stream, timing
// events and per-call scratch.  A context has one (main); a server adds one
// per slot, so that requests run on their own streams.
struct Exec {
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[6] = {};
    double timings[5] = {0, 0, 0, 0, 0};
    std::vector<cudaEvent_t> evpool;                       // per-phase events
    std::vector<cudaEvent_t> kev;                          // start/stop pairs
    std::vector<std::pair<std::string, double>> kev_tag;   // family, work of each pair
    std::map<std::string, KernelStat> kstats;
    DevBuf split_cols, split_colexp;   // split precision: column slices of the current group
    DevBuf split_error;                // bytes 0-15: flags set by a timed-out wait; 16-23: split work counter
    // Page-locked staging for the small uploads of one call (kernel argument
    // arrays), so that they never wait for the stream: reset at the start of
    // each call on this execution state (the previous call has completed).
    char* stage = nullptr;
    size_t stage_bytes = 0, stage_used = 0;
    std::vector<char*> stage_old;  // outgrown blocks, freed when the state is
    double trace_t = 0;            // host time of the last trace mark (SLGPU_HOST_TRACE)
    bool capturing = false;        // launches are being captured into a graph
    // Request arena (serving slots): while arena_on, DevBuf::alloc carves
    // buffers from `arena` (bump allocation, reset per request; the slot's
    // previous request has completed) instead of the stream-ordered pool,
    // whose growth under concurrent streams stalls the launching thread.
    // Allocations that do not fit go to the pool and are counted in
    // arena_miss, by which the arena grows before the next request.
    DevBuf arena;
    size_t arena_off = 0, arena_miss = 0;
    bool arena_on = false;
};

struct Ctx {
    int device = -1;
    int nsm = 0;  // multiprocessors of the device
    bool record_only = false;
    size_t budget = 0;
    int64_t in_use = 0;
    Exec main;
    Exec* x = &main;        // the execution state launches are issued on
    std::recursive_mutex mu;  // one thread at a time inside the context
    std::string last_error;
    int64_t bytes_h2d = 0, bytes_d2h = 0;  // host <-> device bytes copied by the context's calls
    // Tile shapes picked by timing on first use, per contraction kind and
    // group shape {kind (0 split, 1 FP64), tier, ntf, ndof, ngp}: the split
    // kernel's element-tile width NE, the FP64 kernel's rows per block.
    std::map<std::array<int, 5>, int> tile_choice;
    std::map<int, MeshDev> meshes;
    std::map<int, std::unique_ptr<Matrix>> matrices;
    int next_handle = 1;
    std::vector<std::shared_ptr<Pattern>> patterns;  // resident pattern cache
    uint64_t use_clock = 0;
    uint64_t pattern_serial = 0;  // serials handed to the patterns built so far
    DevBuf scratch;  // reusable temporary storage (sort, scans)
    DevBuf hash_acc;
    std::vector<uint8_t> constr_host;  // last constraint array seen by process()
    DevBuf constr_dev;
    uint64_t constr_key[2] = {0, 0};
    int64_t launches = 0;              // kernels launched by this context
    bool graphs = true;                // value-path graphs for process() (slgpu_ctx_set_graphs)
    bool timers = true;                // per-kernel and per-phase events (slgpu_ctx_set_kernel_timers)
    int64_t graph_launches = 0;
    uint64_t next_serial = 1;          // group serial numbers
    std::map<std::string, cudaKernel_t> jit_kernels;  // runtime-compiled coefficient kernels by source
    std::vector<cudaLibrary_t> jit_libs;
    bool jit_broken = false;  // a coefficient kernel failed to compile: interpreter from then on
    std::string jit_error;
    // Page-locked blocks (16 MB, two per copy thread) and events of the
    // pipelined download into pageable host memory (slgpu_matrix_download*).
    static constexpr int kDlStages = 32;
    char* dl_stage[kDlStages] = {};
    cudaEvent_t dl_ev[kDlStages] = {};
    // Page-locked blocks (16 MB, two per copy thread) and events of the
    // pipelined upload of large pageable arrays (group addresses); one upload
    // at a time.
    static constexpr int kUlStages = 16;
    char* ul_stage[kUlStages] = {};
    cudaEvent_t ul_ev[kUlStages] = {};
    std::mutex ul_mu;
    // Record-only contexts: right-hand-side groups and their DOF counts.
    std::vector<std::shared_ptr<GroupDev>> rhs_record;
    std::vector<int64_t> rhs_record_ndofs;
};

// Per-group replacements of the coefficient data for one request (nullptr:
// the group's resident array).
struct GroupData {
    const double* elemdata = nullptr;
    const double* fielddata = nullptr;
    const double* term_scale = nullptr;  // device [nterms], replaces the group's term scales
};

// Whether a group's contraction takes the symmetric form (mirror terms with
// equal scales; engine.cu).
bool group_symmetric(const GroupDev& g);

// Launch pieces of one assembly (engine.cu), issued on ctx->x's stream.
// Whether a step of M at `precision` stores its element matrices as floats:
// FP32-level steps whose groups are all contracted by the split kernels and
// that have no raw fragments.
bool float_values(const Matrix& M, int precision);
std::vector<Segment> build_segments(const Matrix& M, std::vector<int64_t>* group_val_base, int64_t* total_vals, bool f32 = false);
void launch_contractions(Ctx* ctx, const Matrix& M, int precision, const std::vector<int64_t>& gvb, double* vals,
                         const std::vector<GroupData>* ov, bool f32 = false);
std::vector<RowSeg> row_segments(const Matrix& M, const std::vector<Segment>& segs, bool f32 = false);
void launch_row_values(Ctx* ctx, const Matrix& M, Pattern& P, const std::vector<RowSeg>& rsegs, const RowSeg* dsegs, bool rhs,
                       const double* vals, double* Avals, double* Dvals);
// Copies `bytes` from host memory to a new device buffer through the current
// execution state's page-locked staging (asynchronous, stream-ordered).
void upload_staged(Ctx* ctx, DevBuf& buf, const void* src, size_t bytes);
// Copies `bytes` from host memory to existing device memory through the
// current execution state's page-locked staging (asynchronous, stream-ordered).
void upload_staged_into(Ctx* ctx, void* dst, const void* src, size_t bytes);
void stage_reset(Exec& x);
void stage_free(Exec& x);
// Allocations that outlive the current request (per-state scratch kept
// between requests) bypass the arena while one of these is alive.
struct ArenaPause {
    Exec& x;
    bool was;
    explicit ArenaPause(Exec& e) : x(e), was(e.arena_on) { x.arena_on = false; }
    ~ArenaPause() { x.arena_on = was; }
};
int kstat_start(Ctx* ctx, const char* family, double work);
// Records an event on the current execution state's stream (as an event
// node of the graph when the stream is being captured).
void record_event(Ctx* ctx, cudaEvent_t e);
// Host-side launch tracing (SLGPU_HOST_TRACE=1): htrace_begin starts the
// clock of the current execution state; htrace_mark adds the host time since
// the previous mark to `label`.  The totals are printed to stderr at exit.
void htrace_begin(Ctx* ctx);
void htrace_mark(Ctx* ctx, const char* label);
// Split-precision operands of the matrix's groups (built once) and the
// current execution state's split scratch grown to fit them, so that the
// value path allocates nothing for them.
void prepare_value_path(Ctx* ctx, const Matrix& M, int precision);
void kstat_stop(Ctx* ctx, int i);
void kstat_collect(Ctx* ctx);

// Runtime-compiled coefficient kernels (coef_jit.cu).
std::string jit_coef_source(const std::vector<const GroupDev*>& batch);
cudaKernel_t jit_coef_kernel(Ctx* ctx, const std::string& src);
std::vector<char> jit_compile(const std::string& src);  // NVRTC only, no device needed

}  // namespace slgpu
