/* swl_b200 model files: a 2D or 3D session's model as the reference's versioned ASCII VTS model
 * document, and the reader that turns such a file back into session parameters, so that shot
 * requests can be specified by the reference's own model files.
 *
 * Replaces writeModelVts / readModelVts (include/Seis2D/ModelIo2D.hpp:5-16,
 * src/two_d/ModelIo2D.cpp).  The file is byte for byte the reference's for the same session and
 * compute settings; the reader validates the shape, finite data and the FNV-1a checksum, and
 * fails with the reference's messages (swl_last_error()).  Files that ask for the reference's
 * automatic surface-receiver layout (model version 7) are refused: the sessions here take the
 * receiver line as given.
 */
#ifndef SWL_MODELIO_H
#define SWL_MODELIO_H
#include "swl_session.h"
#ifdef __cplusplus
extern "C" {
#endif

/* ModelDocument::compute / backend (ComputeSettings3D, BackendKind3D): recorded in the file. */
typedef struct swl_model_compute {
    int32_t backend;     /* 0 CPU, 1 CUDA */
    int32_t cpu_threads; /* 0 = automatic */
    int32_t cuda_device; /* -1 = largest */
} swl_model_compute;

swl_status swl2d_session_write_model(const swl2d_session *s, const char *path, const swl_model_compute *compute);

typedef struct swl2d_model_document swl2d_model_document;
swl_status swl2d_read_model(const char *path, swl2d_model_document **out);
/* The document's parameters; the layer and surface-sample pointers in *params stay valid until
 * the document is freed.  compute and reference_dt may be null. */
swl_status swl2d_model_document_params(const swl2d_model_document *d, swl_params2d *params, swl_model_compute *compute,
                                       double *reference_dt);
void swl2d_model_document_free(swl2d_model_document *d);

/* The same for 3D: writeModelVts3D / readModelVts3D (include/Seis3D/ModelIo3D.hpp,
 * src/three_d/ModelIo3D.cpp), schema 1 (analytic terrain) or 2 (embedded DEM), layer names kept. */
swl_status swl3d_session_write_model(const swl3d_session *s, const char *path, const swl_model_compute *compute);
typedef struct swl3d_model_document swl3d_model_document;
swl_status swl3d_read_model(const char *path, swl3d_model_document **out);
swl_status swl3d_model_document_params(const swl3d_model_document *d, swl_params3d *params, swl_model_compute *compute,
                                       double *reference_dt);
void swl3d_model_document_free(swl3d_model_document *d);

#ifdef __cplusplus
}
#endif
#endif
