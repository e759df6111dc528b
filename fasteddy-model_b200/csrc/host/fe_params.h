/* fe_params.h -- reader for the FastEddy `name = value # comment` parameter file.
 *
 * Keeps the reference's input format and query semantics so an existing FastEddy
 * parameter file drops in unchanged:
 *   - one `name = value` pair per line, `#` starts a comment, blank values are "absent";
 *   - duplicate names are an error (reference SRC/PARAMETERS/parameters.c:141-146);
 *   - typed queries carry a [min,max] range and a MANDATORY/OPTIONAL status
 *     (reference SRC/PARAMETERS/parameters.c:265-450): an out-of-range value or a
 *     missing mandatory key counts an error, a missing optional key keeps the default;
 *   - keys that no module queried are reported (reference parameters.c:671).
 * Unlike the reference, nothing here calls exit(): every failure is a return code.
 */
#ifndef FE_PARAMS_H
#define FE_PARAMS_H

#ifdef __cplusplus
extern "C" {
#endif

#define FE_PARAM_OK              0
#define FE_PARAM_WARN_DEFAULTED  1000
#define FE_PARAM_ERR_FILE        201
#define FE_PARAM_ERR_FLOAT       203
#define FE_PARAM_ERR_INTEGER     205
#define FE_PARAM_ERR_ABSENT      206
#define FE_PARAM_ERR_DUPLICATE   207
#define FE_PARAM_ERR_SYNTAX      210

#define FE_PARAM_NOT_REQUIRED 0
#define FE_PARAM_OPTIONAL     1
#define FE_PARAM_MANDATORY    2

/* Clear the table and the error count. */
void fe_params_reset(void);
/* Parse a parameter file into the table; returns FE_PARAM_OK or an error code. */
int fe_params_read_file(const char *path);
/* Parse parameter text held in memory (same syntax as the file). */
int fe_params_read_text(const char *text);
int fe_params_query_float(const char *name, float *var, float vmin, float vmax, int req);
int fe_params_query_int(const char *name, int *var, int vmin, int vmax, int req);
/* String values: *out points into the table (NULL when the value is blank or absent). */
int fe_params_query_string(const char *name, const char **out, int req);
/* Number of errors counted by reads and queries since the last reset. */
int fe_params_error_count(void);
/* Write the names of keys present in the file but never queried; returns their count. */
int fe_params_report_unused(char *buf, int buflen);
/* Last error message (for logging from Python). */
const char *fe_params_last_message(void);

#ifdef __cplusplus
}
#endif
#endif
