/* swl_b200 receiver records: SEG-Y export and import, and the reference's receiver CSV files.
 *
 * Replaces the reference's record I/O for downstream tools:
 *   writeSegy / readSegy      (include/SeisCommon/SegyIo.hpp:6-19, src/common/SegyIo.cpp)
 *   2D writeReceivers CSV     (src/two_d/CurvilinearSolver2D.cpp:811-855)
 *   3D writeReceiversCsv      (src/three_d/ReceiverIo.cpp)
 * The files are byte-for-byte those of the reference for the same records and options.
 * Failures return SWL_ERR_INVALID with the reference's message in swl_last_error(); a failed
 * export leaves an existing destination file unchanged (written to a temporary file first).
 */
#ifndef SWL_RECORDS_H
#define SWL_RECORDS_H
#include "swl_b200.h"
#include "swl_session.h"
#ifdef __cplusplus
extern "C" {
#endif

/* One receiver trace (SeisWave::TraceView, include/SeisCommon/SeismicRecords.hpp:9-13). */
typedef struct swl_trace_view {
    double position[3], source[3]; /* metres; z positive down */
    double start_time;             /* seconds (trace delay) */
    const double *channels[3];     /* n_samples values per component, null past n_components */
} swl_trace_view;

/* A record set (SeisWave::RecordDataView, SeismicRecords.hpp:16-29). */
typedef struct swl_record_view {
    const swl_trace_view *traces;
    int32_t n_traces, n_components; /* n_components 1..3 */
    int64_t n_samples;              /* per trace and component */
    const char *components[3];      /* e.g. "Vz", "Vx" */
    double dt;                      /* seconds */
    const char *units;              /* null means "m/s" */
} swl_record_view;

/* SegyExportProfile (SegyIo.hpp:5): rev 2 IEEE32 / IEEE64 with the exact dt, rev 1 IBM32 or IEEE32. */
enum { SWL_SEGY_IEEE32 = 0, SWL_SEGY_IEEE64 = 1, SWL_SEGY_IBM32 = 2, SWL_SEGY_COMPATIBLE_IEEE32 = 3 };

typedef struct swl_segy_options {
    int32_t profile;          /* SWL_SEGY_* */
    double sample_gain;       /* one constant for all traces (> 0); default 1 */
    double sample_interval_s; /* 0 keeps dt; > 0 resamples linearly */
} swl_segy_options;

void swl_segy_options_default(swl_segy_options *o);
/* writeSegy(records, component, path, error, options): one component per file. */
swl_status swl_write_segy(const swl_record_view *records, int32_t component, const char *path, const swl_segy_options *o);

/* readSegy(path, records, error): rev 0/1 and the fixed-header subset of rev 2; IBM, IEEE and
 * integer samples; big or little endian. */
typedef struct swl_segy_records swl_segy_records;
typedef struct swl_segy_info {
    int32_t n_traces;
    int64_t max_samples;
    double dt;
    char component[64], units[64], description[128];
} swl_segy_info;
swl_status swl_read_segy(const char *path, swl_segy_records **out);
void swl_segy_records_free(swl_segy_records *r);
swl_status swl_segy_records_info(const swl_segy_records *r, swl_segy_info *out);
/* Trace `index`: position, source, start time and up to `capacity` samples; *n_samples gets the
 * trace's sample count. */
swl_status swl_segy_records_trace(const swl_segy_records *r, int32_t index, double position[3], double source[3],
                                  double *start_time, double *samples, int64_t capacity, int64_t *n_samples);

/* Sessions.  The record set of a session as the reference's workbench builds it
 * (src/two_d/ui/Workbench2D.cpp:251-268: components Vz, Vx, receivers at (x, 0, z), the source
 * node's coordinates; src/three_d/ui/RecordView3D.cpp:5-6: Vz, Vx, Vy), written as SEG-Y; and
 * the receiver CSV files.  The CSV header's backend line names this library's device. */
swl_status swl2d_session_write_segy(const swl2d_session *s, int32_t component, const char *path, const swl_segy_options *o);
swl_status swl2d_session_write_receivers(const swl2d_session *s, const char *path);
swl_status swl3d_session_write_segy(const swl3d_session *s, int32_t component, const char *path, const swl_segy_options *o);
/* selected[c] for Vx, Vy, Vz (writeReceiversCsv(simulation, path, selected, error)). */
swl_status swl3d_session_write_receivers(const swl3d_session *s, const char *path, const int32_t selected[3]);

#ifdef __cplusplus
}
#endif
#endif
