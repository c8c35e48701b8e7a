/*
 * mjb200: extensions of libmjmlx that have no counterpart in the reference's
 * public headers.  They expose what the B200 engine adds to the method
 * (engine configuration, solver statistics, device-resident stepping,
 * mixed-model batches, the learned Newton warm start) and the compiled-model
 * dump that the FP64 test oracle reads.  Plain C types only.
 */
#ifndef MJB200_H
#define MJB200_H

#include <stddef.h>
#include <stdint.h>

#include "mjmlx.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ model dump */

/* Writes a text dump of the compiled model ("name kind n values..." per line)
 * into buf (NUL-terminated) when bufsize is large enough; returns the number
 * of bytes needed including the NUL, or -1 on a bad handle.  No reference
 * counterpart (the reference hands out the MuJoCo mjModel instead,
 * mjmlx.h:95 mjmlx_get_mj_model). */
MJMLX_API int mjb200_model_dump(const MjmlxModel* model, char* buf, int bufsize);

/* Last error message of the calling thread ("" if none). */
MJMLX_API const char* mjb200_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* MJB200_H */
