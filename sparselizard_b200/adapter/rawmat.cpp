// Replacement for sparselizard's src/formulation/rawmat.cpp (same header,
// rawmat.h, unchanged).  Element contributions recorded by the GPU
// contribution::generate and raw fragments passed to accumulate() are turned
// into the A/D CSR blocks on the device by slgpu_matrix_process, then copied
// into the rawmat's own Arows/Acols/Avals/Drows/Dcols/Dvals members, which
// PETSc borrows exactly as in the reference (MatCreateSeqAIJWithArrays).
#include "rawmat.h"

#include "slgpu_adapter.h"

#include <cstdint>
#include <vector>

namespace {

// Row pointers and column indices of A and D from the last full download,
// with the engine pattern they came from.  indexmat storage is reference
// counted, so the rawmats filled from them share these arrays (PETSc only
// reads them: MatCreateSeqAIJWithArrays borrows them as the structure of a
// matrix whose nonzeros cannot change).  A process() on the same pattern --
// the same serial means the same addresses and constraints -- takes them
// over and downloads the values alone.
struct StructureCache {
    uint64_t serial = 0;
    long long nA = -1, nnzA = -1, nnzD = -1;
    indexmat Arows, Acols, Drows, Dcols;
    indexmat Ainds, Dinds;  // the same serial also means the same constraints
};
StructureCache g_structure;

// Value arrays of A lent to rawmats and taken back when a rawmat is destroyed
// or processed again (only the rawmat uses its Avals; PETSc borrows the
// pointer until the rawmat's destructor).  A buffer that comes back keeps its
// pages, so the next download into it does not fault them in again: on a
// fresh array the first touches, not the link, bound the copy.  The second
// time a buffer is lent it is page-locked (its pages are mapped by then), so
// that downloads go straight into it over the link.  Arrays of at least
// kPooledValues entries are lent; at most kPoolBuffers are kept.
struct ValueBuffer {
    densemat storage;
    long long capacity = 0;
    const rawmat* user = nullptr;
    bool locked = false;
};

void drop_buffer(ValueBuffer& b)
{
    if (b.locked)
        slgpu_host_unregister(slgpu_adapter::context(), b.storage.getvalues());
    b = ValueBuffer();
}
constexpr long long kPooledValues = (long long)1 << 21;
constexpr size_t kPoolBuffers = 2;
std::vector<ValueBuffer> g_values;

densemat lend_values(const rawmat* user, long long n)
{
    if (n < kPooledValues)
        return densemat(n, 1);
    for (ValueBuffer& b : g_values)
        if (b.user == nullptr && b.capacity >= n) {
            b.user = user;
            if (!b.locked)
                b.locked = slgpu_host_register(slgpu_adapter::context(), b.storage.getvalues(), (size_t)b.capacity * sizeof(double)) ==
                           SLGPU_OK;
            return b.storage.getresized(n, 1);
        }
    // A free buffer that is too small is replaced; otherwise one is added
    // while below the limit.
    for (ValueBuffer& b : g_values)
        if (b.user == nullptr) {
            drop_buffer(b);
            b = ValueBuffer{densemat(n, 1), n, user, false};
            return b.storage;
        }
    if (g_values.size() < kPoolBuffers) {
        g_values.push_back(ValueBuffer{densemat(n, 1), n, user, false});
        return g_values.back().storage;
    }
    return densemat(n, 1);
}

void return_values(const rawmat* user)
{
    for (ValueBuffer& b : g_values)
        if (b.user == user)
            b.user = nullptr;
}

}  // namespace

void slgpu_adapter::release_structure_cache(void)
{
    g_structure = StructureCache();
    std::vector<ValueBuffer> kept;
    for (ValueBuffer& b : g_values) {
        if (b.user != nullptr)
            kept.push_back(b);
        else
            drop_buffer(b);
    }
    g_values = kept;
}

rawmat::rawmat(std::shared_ptr<dofmanager> dofmngr)
{
    mydofmanager = dofmngr;
    mymeshnumber = universe::getrawmesh()->getmeshnumber();
}

rawmat::rawmat(std::shared_ptr<dofmanager> dofmngr, Mat inA, Mat inD, indexmat inAinds, indexmat inDinds)
{
    mydofmanager = dofmngr;
    Amat = inA;
    Dmat = inD;
    Ainds = inAinds;
    Dinds = inDinds;
    mymeshnumber = universe::getrawmesh()->getmeshnumber();
}

rawmat::~rawmat(void)
{
    slgpu_adapter::forget_matrix(this);
    return_values(this);
    // PETSc objects may only be destroyed before PetscFinalize.
    PetscBool ispetscinitialized;
    PetscInitialized(&ispetscinitialized);
    if (ispetscinitialized == PETSC_TRUE) {
        if (Amat != PETSC_NULLPTR)
            MatDestroy(&Amat);
        if (Dmat != PETSC_NULLPTR)
            MatDestroy(&Dmat);
        if (isitfactored)
            KSPDestroy(&myksp);
    }
}

long long int rawmat::countrows(void) { return mydofmanager == NULL ? 0 : mydofmanager->countdofs(); }

long long int rawmat::countcolumns(void) { return mydofmanager == NULL ? 0 : mydofmanager->countdofs(); }

void rawmat::accumulate(indexmat rowadresses, indexmat coladresses, densemat vals)
{
    // Host fragments (ports, mat(...) constructors) are kept as in the
    // reference and shipped to the device when the matrix is processed.
    if (vals.count() > 0) {
        accumulatedrowindices.push_back(rowadresses);
        accumulatedcolindices.push_back(coladresses);
        accumulatedvals.push_back(vals);
    }
}

void rawmat::process(std::vector<bool>& isconstrained)
{
    const long long ndofs = countrows();

    slgpu_ctx* ctx = slgpu_adapter::context();
    int handle = slgpu_adapter::matrix_handle(this, ndofs);
    for (size_t i = 0; i < accumulatedvals.size(); i++) {
        slgpu_adapter::check(slgpu_matrix_add_fragment(ctx, handle, accumulatedrowindices[i].countrows(),
                                                       accumulatedcolindices[i].countrows(), accumulatedvals[i].countrows(),
                                                       accumulatedvals[i].countcolumns(), accumulatedrowindices[i].getvalues(),
                                                       accumulatedcolindices[i].getvalues(), accumulatedvals[i].getvalues()),
                             "slgpu_matrix_add_fragment");
    }
    std::vector<uint8_t> constr((size_t)ndofs);
#pragma omp parallel for schedule(static) if (ndofs > (1 << 16))
    for (long long i = 0; i < ndofs; i++) constr[i] = isconstrained[i] ? 1 : 0;

    slgpu_csr_info info{};
    slgpu_adapter::set_last_processed(this);
    slgpu_adapter::check(slgpu_matrix_process(ctx, handle, constr.data(), slgpu_adapter::precision(), &info), "slgpu_matrix_process");
    slgpu_adapter::addresses_processed(this);
    nnzA = info.nnzA;
    nnzD = info.nnzD;

    uint64_t serial = 0;
    slgpu_adapter::check(slgpu_matrix_pattern_serial(ctx, handle, &serial), "slgpu_matrix_pattern_serial");
    return_values(this);
    Avals = lend_values(this, nnzA);
    Dvals = densemat(nnzD, 1);
    StructureCache& sc = g_structure;
    if (serial != 0 && sc.serial == serial && sc.nA == info.nA && sc.nnzA == nnzA && sc.nnzD == nnzD) {
        Ainds = sc.Ainds;
        Dinds = sc.Dinds;
        Arows = sc.Arows;
        Acols = sc.Acols;
        Drows = sc.Drows;
        Dcols = sc.Dcols;
        slgpu_adapter::check(slgpu_matrix_download_values(ctx, handle, Avals.getvalues(), Dvals.getvalues()),
                             "slgpu_matrix_download_values");
    } else {
        std::vector<int> renumtolocalindex;
        gentools::findtruefalse(isconstrained, Dinds, Ainds, renumtolocalindex);
        Arows = indexmat(Ainds.count() + 1, 1);
        Acols = indexmat(nnzA, 1);
        Drows = indexmat(Ainds.count() + 1, 1);
        Dcols = indexmat(nnzD, 1);
        slgpu_adapter::check(slgpu_matrix_download(ctx, handle, Arows.getvalues(), Acols.getvalues(), Avals.getvalues(),
                                                   Drows.getvalues(), Dcols.getvalues(), Dvals.getvalues()),
                             "slgpu_matrix_download");
        sc = StructureCache();
        sc.serial = serial;
        sc.nA = Ainds.count();
        sc.nnzA = nnzA;
        sc.nnzD = nnzD;
        sc.Arows = Arows;
        sc.Acols = Acols;
        sc.Drows = Drows;
        sc.Dcols = Dcols;
        sc.Ainds = Ainds;
        sc.Dinds = Dinds;
    }

    MatCreateSeqAIJWithArrays(PETSC_COMM_SELF, Ainds.count(), Ainds.count(), Arows.getvalues(), Acols.getvalues(), Avals.getvalues(), &Amat);
    MatAssemblyBegin(Amat, MAT_FINAL_ASSEMBLY);
    MatAssemblyEnd(Amat, MAT_FINAL_ASSEMBLY);

    MatCreateSeqAIJWithArrays(PETSC_COMM_SELF, Ainds.count(), Dinds.count(), Drows.getvalues(), Dcols.getvalues(), Dvals.getvalues(), &Dmat);
    MatAssemblyBegin(Dmat, MAT_FINAL_ASSEMBLY);
    MatAssemblyEnd(Dmat, MAT_FINAL_ASSEMBLY);
}

void rawmat::clearfragments(void)
{
    accumulatedrowindices = {};
    accumulatedcolindices = {};
    accumulatedvals = {};
    slgpu_adapter::release_matrix(this);
}

void rawmat::print(void)
{
    std::cout << std::endl;
    if (mydofmanager == NULL)
        std::cout << "Undefined matrix" << std::endl;
    else if (countrows() > 0) {
        std::cout << "A block " << Ainds.count() << "x" << Ainds.count() << ":" << std::endl << std::endl;
        MatView(Amat, PETSC_VIEWER_STDOUT_SELF);
        std::cout << std::endl << "D block " << Ainds.count() << "x" << Dinds.count() << ":" << std::endl << std::endl;
        MatView(Dmat, PETSC_VIEWER_STDOUT_SELF);
    } else
        std::cout << "Empty matrix" << std::endl;
    std::cout << std::endl;
}

std::shared_ptr<rawmat> rawmat::extractaccumulated(void)
{
    std::shared_ptr<rawmat> output(new rawmat(mydofmanager));
    output->accumulatedrowindices = accumulatedrowindices;
    output->accumulatedcolindices = accumulatedcolindices;
    output->accumulatedvals = accumulatedvals;
    slgpu_adapter::share_matrix(this, output.get());
    return output;
}

indexmat rawmat::getainds(void) { return Ainds; }
indexmat rawmat::getdinds(void) { return Dinds; }
Mat rawmat::getapetsc(void) { return Amat; }
Mat rawmat::getdpetsc(void) { return Dmat; }
std::shared_ptr<dofmanager> rawmat::getdofmanager(void) { return mydofmanager; }
KSP* rawmat::getksp(void) { return &myksp; }
