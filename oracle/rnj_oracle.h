/* rnj_oracle.h -- CPU restatement of rapidNJ's distance path (test infrastructure
 * only; see rnj_oracle.c for the reference lines each function follows). */
#ifndef RNJ_ORACLE_H
#define RNJ_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_DNA = 0, ORC_PROTEIN = 1 };
enum { ORC_JC = 0, ORC_KIMURA = 1 };

int orc_detect_type(const char *seq0, int L);
char orc_resolve_char(char c, int type);
int orc_pam_value(int idx);
uint64_t orc_protein_fast_valid(uint64_t valid, int L);

void orc_pair_counts(const char *a, const char *b, int L, int type, int naive, uint64_t out[3]);
/* seqs: n*L bytes row-major.  out: n*n*3 uint32, filled for j>i (or every j when full). */
void orc_counts(const char *seqs, int n, int L, int type, int naive, int full, uint32_t *out);
void orc_counts_rows(const char *seqs, int n, int L, int type, int naive, int full, int row0,
                     int row1, uint32_t *out);

float orc_jc(uint64_t c0, uint64_t c1, uint64_t valid, int type);
float orc_k2p(uint64_t ts, uint64_t tv, uint64_t valid);
float orc_kimura_protein(uint64_t mism, uint64_t valid);
double orc_jc_d(uint64_t c0, uint64_t c1, uint64_t valid, int type);
double orc_k2p_d(uint64_t ts, uint64_t tv, uint64_t valid);
double orc_kimura_protein_d(uint64_t mism, uint64_t valid);
double orc_matrix_d(const uint32_t *counts, int n, int L, int type, int model, int naive,
                    int compat_wrap, int full, double *out);
float orc_distance(const uint32_t c[3], int L, int type, int model, int naive, int compat_wrap);

/* Post-processed n*n float matrix from upper-triangle counts; returns the max. */
float orc_matrix(const uint32_t *counts, int n, int L, int type, int model, int naive,
                 int compat_wrap, float *out);
float orc_matrix_full(const uint32_t *counts, int n, int L, int type, int model, int naive,
                      int compat_wrap, float *out);

/* Pre-post-process distances (saturated = -1) for j > i, or every pair when full. */
void orc_raw_distances(const uint32_t *counts, int n, int L, int type, int model, int naive,
                       int compat_wrap, int full, float *out);

#ifdef __cplusplus
}
#endif
#endif
