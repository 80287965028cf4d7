/*
 * Stand-in for an htslib header (TEST INFRASTRUCTURE ONLY). htslib, a git submodule of
 * the reference, is absent; impl/polisher.c reaches it only through declarations in
 * inc/htsIntegration.h and the samtools bed index header, which name these types.
 */
#ifndef MP_HTSLIB_NAMES_HTS_H_
#define MP_HTSLIB_NAMES_HTS_H_
typedef struct bam1_t bam1_t;
typedef struct hts_reglist_t hts_reglist_t;
#endif
