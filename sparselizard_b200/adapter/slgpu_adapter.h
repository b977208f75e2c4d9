// Glue between sparselizard's host objects and the slgpu C ABI.
//
// Used by the two translation units that replace sparselizard's
// src/formulation/contribution.cpp and src/formulation/rawmat.cpp.  The
// class headers (contribution.h, rawmat.h) are unchanged, so per-rawmat
// engine state lives in a side table keyed by the rawmat address.
#ifndef SLGPU_ADAPTER_H
#define SLGPU_ADAPTER_H

#include "slgpu.h"
#include "indexmat.h"

#include <memory>
#include <string>

class rawmat;
class expression;

namespace slgpu_adapter {

// The process-wide engine context (device 0, or record-only when the
// environment variable SLGPU_RECORD_ONLY=1).  Raises through logs::error when
// no CUDA device is usable: there is no CPU fallback.
slgpu_ctx* context(void);

// Contraction precision from SLGPU_PRECISION (fp64 | split | fp32), default fp64.
int precision(void);

// Throws a sparselizard error (std::runtime_error via logs) when status != 0.
void check(int status, const char* what);

// Makes sure the current mesh's nodes and the curved-node connectivity of
// element type `elemtype` are resident; returns the engine mesh id.
int ensure_mesh(int elemtype);

// Engine matrix handle owned by a rawmat (created on first use, with address
// sharing on: slgpu_matrix_share_addresses).
int matrix_handle(rawmat* m, long long ndofs);
// Keeps an address array given to the rawmat's engine matrix alive until
// addresses_processed(m), which rawmat::process calls after
// slgpu_matrix_process (the engine may reuse its device copy until then).
void keep_addresses(rawmat* m, const indexmat& a);
void addresses_processed(rawmat* m);
// Handle if any (0 = none).
int find_matrix_handle(rawmat* m);
// Moves/copies ownership of the engine matrix between rawmats.
void share_matrix(rawmat* from, rawmat* to);
// Forgets a rawmat's engine matrix (destroying it when no other rawmat uses it).
void release_matrix(rawmat* m);
// Drops every engine matrix tied to a rawmat (its destructor).
void forget_matrix(rawmat* m);

// True on a record-only context (SLGPU_RECORD_ONLY=1): groups are recorded for
// inspection and every assembly request ends in an error.
bool record_only(void);
// Remembers the engine matrix handed to the last rawmat::process call.
void set_last_processed(rawmat* m);

// Forgets the DOF addresses kept for the contributions of later assemblies
// (contribution.cpp).
void clear_address_cache(void);

// rawmat::process keeps the host CSR structure (Arows, Acols, Drows, Dcols)
// of the last pattern it downloaded and shares it with the next rawmat
// processed on the same engine pattern, which then downloads only values; it
// also keeps up to two value arrays of A that rawmats gave back, to download
// into pages that are already mapped.  This frees what is kept and not in use
// (the rawmats using an array keep it).
void release_structure_cache(void);

// Integral of a scalar expression over a physical region at a Gauss order
// (what expression::integrate computes, src/expression/expression.cpp:808-889)
// on the GPU: the expression is lowered to a coefficient program, evaluated
// at the Gauss points with its weights and |det J| per element, and summed.
// Field values inside the expression are interpolated on the device
// (rawfield::interpolate, src/field/rawfield.cpp:2632-2686).
double integrate(expression e, int physreg, int integrationorder);

}  // namespace slgpu_adapter

extern "C" {
// Context and last processed matrix handle of this process (inspection of
// record-only runs).
slgpu_ctx* slgpu_adapter_ctx(void);
int slgpu_adapter_last_handle(void);
}

#endif
