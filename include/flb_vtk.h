/* flb_vtk.h -- VTK output of device-resident fields (libflb_b200.so).
 *
 * The reference writes fields with its vtmo writers (src/io/vtm_writer.h:
 * 288-663, vtmo::vtmWriter with ScalarWriter / VectorWriter / PhysScalarWriter
 * / PhysVectorWriter over vtino::vtiManager, src/io/vti_writer.h:424-986):
 * per block one .vti file whose <DataArray ... encoding="base64"> bodies are
 * produced by Base64Encoder (src/io/base64.h).  This entry point produces such
 * a body on the GPU -- crop, type conversion, optional unit conversion and
 * base64 in one kernel -- so that only the text crosses to the host; the
 * C++ host classes (freelb_b200/cpp/freelb.h, namespace vtmo) write the XML
 * around it exactly as the reference does.  Conventions as in flb.h.
 */
#ifndef FLB_VTK_H_
#define FLB_VTK_H_

#include "flb.h"

#ifdef __cplusplus
extern "C" {
#endif

/* field: FLB_FIELD_RHO / FLB_FIELD_VELOCITY / FLB_FIELD_ALPHA (arithmetic type
 * of the lattice: FP64 storage -> double, else float), or FLB_VTK_FLAG (the
 * uint8 flags). */
#define FLB_VTK_FLAG 16

/* Base64 body of one DataArray of block `block`: the cells [overlap, n -
 * overlap) on each axis, x fastest, VELOCITY components interleaved,
 * converted to `out_dtype` (FLB_DTYPE_F32 / FLB_DTYPE_F64; ignored for
 * FLB_VTK_FLAG, which stays UInt8), and, when `map` is non-zero, each value v
 * replaced by v * scale + offset evaluated in the field's type first (the
 * Phys writers' unit conversion; offset 0 skips the addition).  The body is
 * the 4-byte size (unsigned int, bytes of data) base64-encoded on its own
 * followed by the base64 of the data, exactly the characters the reference
 * writes between the DataArray tags (without the newline after them).
 * `*len` receives the number of characters; with out == NULL only the length
 * is computed, else `cap` must be at least that.  `stream` orders the work
 * and is synchronised before returning. */
FLB_API int flb_vtk_field_base64(flb_lattice* lat, int block, int field, int overlap,
                                 int out_dtype, int map, double scale, double offset, char* out,
                                 size_t cap, size_t* len, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FLB_VTK_H_ */
