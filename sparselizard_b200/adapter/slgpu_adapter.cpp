// Process-wide glue for the sparselizard adapter: engine context, resident
// mesh geometry and the rawmat -> engine matrix side table.
#include "slgpu_adapter.h"

#include "element.h"
#include "elements.h"
#include "logs.h"
#include "nodes.h"
#include "rawmesh.h"
#include "universe.h"

#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

namespace slgpu_adapter {

namespace {

slgpu_ctx* g_ctx = nullptr;
bool g_ctx_failed = false;
bool g_record_only = false;
int g_last_handle = 0;

struct MatEntry {
    int handle = 0;
    // Address arrays given to the engine matrix since its last process(): the
    // engine reuses the device copy of an array it has seen before (same host
    // pointer and length), so none of them may be freed, and its address
    // reused for other values, before process().
    std::vector<indexmat> addresses;
    ~MatEntry()
    {
        if (handle != 0 && g_ctx != nullptr)
            slgpu_matrix_destroy(g_ctx, handle);
    }
};
std::map<rawmat*, std::shared_ptr<MatEntry>> g_mats;
std::shared_ptr<MatEntry> g_last_entry;
std::map<rawmat*, std::shared_ptr<MatEntry>> g_processed;

// One engine mesh per sparselizard mesh -- the rawmesh object together with
// its number, which only counts adaptations of one loaded mesh -- so that
// matrices assembled on earlier meshes stay valid as templates after another
// mesh is loaded.  A mesh whose nodes move in place is updated in place.
struct MeshState {
    int id = 0;  // engine mesh id
    long long nnodes = -1;
    unsigned long long coordhash = 0;
    std::map<int, long long> typecounts;  // element type -> uploaded count
};
std::map<std::pair<const void*, int>, MeshState> g_meshes;  // by (rawmesh, number)

struct CtxGuard {
    ~CtxGuard()
    {
        g_mats.clear();
        g_processed.clear();
        g_last_entry.reset();
        if (g_ctx != nullptr)
            slgpu_ctx_destroy(g_ctx);
        g_ctx = nullptr;
    }
} g_guard;

[[noreturn]] void raise(const std::string& msg)
{
    logs log;
    log.msg() << "Error in the GPU assembly engine: " << msg << std::endl;
    log.error();
    throw std::runtime_error(msg);  // not reached: logs::error throws
}

}  // namespace

slgpu_ctx* context(void)
{
    if (g_ctx != nullptr)
        return g_ctx;
    if (g_ctx_failed)
        raise("no usable CUDA device (earlier initialisation failed)");
    const char* rec = std::getenv("SLGPU_RECORD_ONLY");
    unsigned flags = (rec != nullptr && std::strcmp(rec, "1") == 0) ? SLGPU_CTX_RECORD_ONLY : 0u;
    g_record_only = flags != 0;
    size_t budget = 0;
    if (const char* b = std::getenv("SLGPU_HBM_BUDGET_GB"))
        budget = (size_t)(std::atof(b) * 1e9);
    int device = 0;
    if (const char* d = std::getenv("SLGPU_DEVICE"))
        device = std::atoi(d);
    int st = slgpu_ctx_create(device, budget, flags, &g_ctx);
    if (st != SLGPU_OK) {
        g_ctx = nullptr;
        g_ctx_failed = true;
        raise("cannot create a device context on CUDA device 0 (status " + std::to_string(st) +
              "); this build of sparselizard assembles on the GPU only");
    }
    return g_ctx;
}

int precision(void)
{
    const char* p = std::getenv("SLGPU_PRECISION");
    if (p == nullptr || std::strcmp(p, "fp64") == 0)
        return SLGPU_PREC_FP64;
    if (std::strcmp(p, "split") == 0)
        return SLGPU_PREC_SPLIT;
    if (std::strcmp(p, "fp32") == 0)
        return SLGPU_PREC_FP32;
    raise(std::string("unknown SLGPU_PRECISION '") + p + "' (fp64, split or fp32)");
}

void check(int status, const char* what)
{
    if (status == SLGPU_OK)
        return;
    char buf[1024] = {0};
    if (g_ctx != nullptr)
        slgpu_last_error(g_ctx, buf, sizeof(buf));
    raise(std::string(what) + " failed (status " + std::to_string(status) + "): " + buf);
}

int ensure_mesh(int elemtype)
{
    slgpu_ctx* ctx = context();
    std::shared_ptr<rawmesh> rm = universe::getrawmesh();
    nodes* nd = rm->getnodes();
    std::vector<double>* xyz = nd->getcoordinates();
    long long nn = (long long)xyz->size() / 3;
    // Cheap content hash of the coordinates (meshes can move in place), in
    // four interleaved chains so that their multiplies overlap.
    const unsigned long long* words = reinterpret_cast<const unsigned long long*>(xyz->data());
    const size_t nw = xyz->size();
    unsigned long long c[4] = {1469598103934665603ull, 1099511628211ull, 0x9E3779B97F4A7C15ull, 0xD6E8FEB86659FD93ull};
    size_t i = 0;
    for (; i + 4 <= nw; i += 4) {
        c[0] = (c[0] ^ words[i]) * 1099511628211ull;
        c[1] = (c[1] ^ words[i + 1]) * 1099511628211ull;
        c[2] = (c[2] ^ words[i + 2]) * 1099511628211ull;
        c[3] = (c[3] ^ words[i + 3]) * 1099511628211ull;
    }
    for (; i < nw; i++) c[0] = (c[0] ^ words[i] ^ i) * 1099511628211ull;
    unsigned long long h = 1469598103934665603ull;
    for (int k = 0; k < 4; k++) h = (h ^ c[k]) * 1099511628211ull;
    const std::pair<const void*, int> key(rm.get(), rm->getmeshnumber());
    auto mit = g_meshes.find(key);
    if (mit == g_meshes.end()) {
        MeshState st;
        st.id = (int)g_meshes.size();
        mit = g_meshes.emplace(key, st).first;
    }
    MeshState& g_mesh = mit->second;
    if (g_mesh.nnodes != nn || g_mesh.coordhash != h) {
        check(slgpu_mesh_set_nodes(ctx, g_mesh.id, nn, xyz->data()), "slgpu_mesh_set_nodes");
        g_mesh.nnodes = nn;
        g_mesh.coordhash = h;
        g_mesh.typecounts.clear();
    }
    elements* els = rm->getelements();
    long long ne = els->count(elemtype);
    auto it = g_mesh.typecounts.find(elemtype);
    if (it == g_mesh.typecounts.end() || it->second != ne) {
        element el(elemtype, els->getcurvatureorder());
        int ncn = el.countcurvednodes();
        std::vector<int32_t> conn((size_t)ne * ncn);
        for (long long e = 0; e < ne; e++)
            for (int k = 0; k < ncn; k++) conn[(size_t)e * ncn + k] = els->getsubelement(0, elemtype, (int)e, k);
        check(slgpu_mesh_set_elements(ctx, g_mesh.id, elemtype, ncn, ne, conn.data()), "slgpu_mesh_set_elements");
        g_mesh.typecounts[elemtype] = ne;
    }
    return g_mesh.id;
}

int find_matrix_handle(rawmat* m)
{
    auto p = g_processed.find(m);
    if (p != g_processed.end())
        return p->second->handle;
    auto it = g_mats.find(m);
    return it == g_mats.end() ? 0 : it->second->handle;
}

int matrix_handle(rawmat* m, long long ndofs)
{
    slgpu_ctx* ctx = context();
    auto it = g_mats.find(m);
    if (it == g_mats.end()) {
        auto e = std::make_shared<MatEntry>();
        check(slgpu_matrix_create(ctx, ndofs, &e->handle), "slgpu_matrix_create");
        check(slgpu_matrix_share_addresses(ctx, e->handle, 1), "slgpu_matrix_share_addresses");
        g_mats[m] = e;
        return e->handle;
    }
    if (it->second.use_count() > 1) {
        // Shared with another rawmat (extractaccumulated): copy before writing.
        auto e = std::make_shared<MatEntry>();
        check(slgpu_matrix_clone(ctx, it->second->handle, &e->handle), "slgpu_matrix_clone");
        e->addresses = it->second->addresses;
        it->second = e;
    }
    return it->second->handle;
}

void keep_addresses(rawmat* m, const indexmat& a)
{
    auto it = g_mats.find(m);
    if (it != g_mats.end())
        it->second->addresses.push_back(a);
}

void addresses_processed(rawmat* m)
{
    auto it = g_mats.find(m);
    if (it != g_mats.end())
        it->second->addresses.clear();
}

void share_matrix(rawmat* from, rawmat* to)
{
    auto it = g_mats.find(from);
    if (it != g_mats.end())
        g_mats[to] = it->second;
}

void release_matrix(rawmat* m) { g_mats.erase(m); }

void forget_matrix(rawmat* m)
{
    g_mats.erase(m);
    g_processed.erase(m);
}

bool record_only(void)
{
    context();
    return g_record_only;
}

void set_last_processed(rawmat* m)
{
    // Keeps the engine matrix alive after the rawmat is gone, so that a
    // record-only run can be inspected once sparselizard has raised.
    auto it = g_mats.find(m);
    g_last_entry = it == g_mats.end() ? nullptr : it->second;
    g_last_handle = g_last_entry ? g_last_entry->handle : 0;
    // The processed engine matrix (resident pattern and values) stays with
    // the rawmat until it is destroyed, even after clearfragments().
    if (g_last_entry)
        g_processed[m] = g_last_entry;
}

}  // namespace slgpu_adapter

extern "C" slgpu_ctx* slgpu_adapter_ctx(void) { return slgpu_adapter::g_ctx; }
extern "C" int slgpu_adapter_last_handle(void) { return slgpu_adapter::g_last_handle; }
