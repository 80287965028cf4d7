/*
 * POA ORACLE harness -- TEST INFRASTRUCTURE ONLY.
 *
 * Links against the reference's own impl/polisher.c (with impl/pairwiseAligner.c and
 * impl/stateMachine.c), compiled unmodified from the reference tree by oracle/Makefile
 * (output: oracle/_ref/libref_poa.so), and exposes the POA steps of the polishing loop
 * (poa_realign, poa_getConsensus, poa_getAnchorAlignments,
 * poa_estimateRepeatCountsUsingBayesianModel, poa_realignIterative / poa_realignAll in
 * consensus mode) through plain pointers, so the tests can compare the library's POA
 * loop with the reference's node weights, indels, anchors and consensus. Only tests/
 * load it, as the checker.
 *
 * impl/bubbleGraph.c is compiled in as well, so the polish mode of the loop (poa_polish:
 * bubbleGraph_constructFromPoa, the allele choice and the new consensus string) runs as the
 * reference wrote it; its bubbles, read substrings, alleles and allele supports are exported
 * for the tests. The diploid phasing functions that file also holds call into impl/hmm.c and
 * its neighbours, which are not compiled: their stand-ins below abort.
 */
#include "margin.h"

/* accessors of oracle/ref_harness.c (compiled into the same library) */
typedef struct {
    double threshold;
    int64_t minDiagsBetweenTraceBack;
    int64_t traceBackDiagonals;
    int64_t diagonalExpansion;
    int64_t constraintDiagonalTrim;
    int64_t splitMatrixBiggerThanThis;
    int64_t dynamicAnchorExpansion;
    double gapGamma;
} RefoParams;
PairwiseAlignmentParameters *refo_params_to_reference(const RefoParams *q);
StateMachine *refo_model_state_machine(void *handle);
RepeatSubMatrix *refo_model_repeat_matrix(void *handle);

/* defined in impl/polisher.c without a prototype in inc/margin.h */
double poa_getTotalErrorWeight(Poa *poa);

/* ---- phasing functions named by impl/bubbleGraph.c: the diploid phasing (impl/hmm.c and
 * its neighbours) is not part of this oracle, so these stand-ins abort if ever reached ---- */
#define PHASING_ONLY(name) st_errAbort("%s: phasing is not part of the POA oracle", name)

stGenomeFragment *stGenomeFragment_construct(stRPHmm *hmm, stList *path) {
    (void) hmm, (void) path;
    PHASING_ONLY("stGenomeFragment_construct");
    return NULL;
}
stGenomeFragment *stGenomeFragment_constructEmpty(stReference *ref, uint64_t refStart, uint64_t length, stSet *reads1,
                                                  stSet *reads2) {
    (void) ref, (void) refStart, (void) length, (void) reads1, (void) reads2;
    PHASING_ONLY("stGenomeFragment_constructEmpty");
    return NULL;
}
void stGenomeFragment_refineGenomeFragment(stGenomeFragment *gF, stRPHmm *hmm, stList *path, int64_t maxIterations) {
    (void) gF, (void) hmm, (void) path, (void) maxIterations;
    PHASING_ONLY("stGenomeFragment_refineGenomeFragment");
}
stProfileSeq *stProfileSeq_constructEmptyProfile(stReference *ref, char *readId, int64_t referenceStart,
                                                 int64_t length) {
    (void) ref, (void) readId, (void) referenceStart, (void) length;
    PHASING_ONLY("stProfileSeq_constructEmptyProfile");
    return NULL;
}
void stProfileSeq_destruct(stProfileSeq *seq) {
    (void) seq;
    PHASING_ONLY("stProfileSeq_destruct");
}
void stRPHmm_forwardBackward(stRPHmm *hmm) {
    (void) hmm;
    PHASING_ONLY("stRPHmm_forwardBackward");
}
stList *stRPHmm_forwardTraceBack(stRPHmm *hmm) {
    (void) hmm;
    PHASING_ONLY("stRPHmm_forwardTraceBack");
    return NULL;
}
stList *getRPHmms(stList *profileSeqs, stRPHmmParameters *params) {
    (void) profileSeqs, (void) params;
    PHASING_ONLY("getRPHmms");
    return NULL;
}
stList *filterReadsByCoverageDepth(stList *profileSeqs, stRPHmmParameters *params, stList *filteredProfileSeqs,
                                   stList *discardedProfileSeqs) {
    (void) profileSeqs, (void) params, (void) filteredProfileSeqs, (void) discardedProfileSeqs;
    PHASING_ONLY("filterReadsByCoverageDepth");
    return NULL;
}
stRPHmm *fuseTilingPath(stList *tilingPath) {
    (void) tilingPath;
    PHASING_ONLY("fuseTilingPath");
    return NULL;
}
stList *mergeTwoTilingPaths(stList *tilingPath1, stList *tilingPath2) {
    (void) tilingPath1, (void) tilingPath2;
    PHASING_ONLY("mergeTwoTilingPaths");
    return NULL;
}
double getLogProbOfReadGivenHaplotype(uint64_t *haplotypeString, int64_t start, int64_t length,
                                      stProfileSeq *profileSeq, stReference *ref) {
    (void) haplotypeString, (void) start, (void) length, (void) profileSeq, (void) ref;
    PHASING_ONLY("getLogProbOfReadGivenHaplotype");
    return 0.0;
}
int popcount64(uint64_t x) {
    (void) x;
    PHASING_ONLY("popcount64");
    return 0;
}

/* ---- construction ---- */

static RleString *makeRle(const char *chars, const uint32_t *counts, int64_t n) {
    RleString *r = st_calloc(1, sizeof(RleString));
    r->length = (uint64_t) n;
    r->rleString = st_calloc(n + 1, 1);
    r->repeatCounts = st_calloc(n > 0 ? n : 1, sizeof(uint64_t));
    for (int64_t i = 0; i < n; i++) {
        r->rleString[i] = chars[i];
        r->repeatCounts[i] = counts[i];
        r->nonRleLength += counts[i];
    }
    return r;
}

/* PolishParams for the consensus-mode loop; anchorProbs is the
 * minPosteriorProbForAlignmentAnchors array (pairs of probability, expansion). */
void *refpoa_params_create(void *modelFwd, void *modelRev, const RefoParams *ap, int useRle, double referencePenalty,
                           int compareRepeatCounts, const double *anchorProbs, int64_t nAnchorProbs,
                           int64_t minIterations, int64_t maxIterations) {
    PolishParams *pp = st_calloc(1, sizeof(PolishParams));
    pp->useRunLengthEncoding = useRle != 0;
    pp->useRepeatCountsInAlignment = useRle != 0;
    pp->alphabet = alphabet_constructNucleotide();
    pp->stateMachineForForwardStrandRead = refo_model_state_machine(modelFwd);
    pp->stateMachineForReverseStrandRead = refo_model_state_machine(modelRev);
    pp->p = refo_params_to_reference(ap);
    pp->repeatSubMatrix = refo_model_repeat_matrix(modelFwd);
    pp->referenceBasePenalty = referencePenalty;
    pp->poaConstructCompareRepeatCounts = compareRepeatCounts != 0;
    pp->minPosteriorProbForAlignmentAnchors = st_calloc(nAnchorProbs, sizeof(double));
    memcpy(pp->minPosteriorProbForAlignmentAnchors, anchorProbs, sizeof(double) * nAnchorProbs);
    pp->minPosteriorProbForAlignmentAnchorsLength = nAnchorProbs;
    pp->minPoaConsensusIterations = (uint64_t) minIterations;
    pp->maxPoaConsensusIterations = (uint64_t) maxIterations;
    pp->minRealignmentPolishIterations = 0;
    pp->maxRealignmentPolishIterations = 0;
    return pp;
}

void refpoa_params_destroy(void *handle) {
    PolishParams *pp = handle;
    if (pp == NULL) {
        return;
    }
    alphabet_destruct(pp->alphabet);
    pairwiseAlignmentBandingParameters_destruct(pp->p);
    free(pp->minPosteriorProbForAlignmentAnchors);
    free(pp);
}

/* The polish-mode parameters of poa_polish (impl/bubbleGraph.c:800-978) and the number of
 * polish iterations poa_realignAll runs after the consensus iterations (impl/polisher.c:2123-2126). */
void refpoa_params_set_polish(void *handle, int useReadAlleles, double candidateVariantWeight, int64_t columnAnchorTrim,
                              int64_t filterReadsWhileHaveAtLeastThisCoverage, double minAvgBaseQuality,
                              int64_t maxConsensusStrings, int64_t minPolishIterations, int64_t maxPolishIterations) {
    PolishParams *pp = handle;
    pp->useReadAlleles = useReadAlleles != 0;
    pp->candidateVariantWeight = candidateVariantWeight;
    pp->columnAnchorTrim = (uint64_t) columnAnchorTrim;
    pp->filterReadsWhileHaveAtLeastThisCoverage = (uint64_t) filterReadsWhileHaveAtLeastThisCoverage;
    pp->minAvgBaseQuality = minAvgBaseQuality;
    pp->maxConsensusStrings = (uint64_t) maxConsensusStrings;
    pp->minRealignmentPolishIterations = (uint64_t) minPolishIterations;
    pp->maxRealignmentPolishIterations = (uint64_t) maxPolishIterations;
}

static void readDestruct(void *p) {
    BamChunkRead *r = p;
    rleString_destruct(r->rleRead);
    free(r->qualities);
    free(r);
}

/* Reads: run-length strings laid end to end (chars, counts), offsets[n+1], strand[n]. */
void *refpoa_reads_create(int64_t n, const char *chars, const uint32_t *counts, const int64_t *offsets,
                          const uint8_t *strand) {
    stList *reads = stList_construct3(0, readDestruct);
    for (int64_t i = 0; i < n; i++) {
        BamChunkRead *r = st_calloc(1, sizeof(BamChunkRead));
        r->rleRead = makeRle(chars + offsets[i], counts + offsets[i], offsets[i + 1] - offsets[i]);
        r->forwardStrand = strand[i] != 0;
        stList_append(reads, r);
    }
    return reads;
}

/* Per-run quality values of every read (the run-length form rleString_rleQualities makes,
 * impl/polisher.c:1692-1714), laid end to end like the reads' runs. */
void refpoa_reads_set_qualities(void *reads, const uint8_t *qualities, const int64_t *offsets) {
    for (int64_t i = 0; i < stList_length(reads); i++) {
        BamChunkRead *r = stList_get(reads, i);
        free(r->qualities);
        int64_t n = offsets[i + 1] - offsets[i];
        r->qualities = st_calloc(n > 0 ? n : 1, 1);
        memcpy(r->qualities, qualities + offsets[i], (size_t) n);
    }
}

void refpoa_reads_destroy(void *reads) {
    stList_destruct(reads);
}

/* Anchor alignments: per read, triples (x, y, expansion) in reference coordinates. */
void *refpoa_anchors_create(int64_t n, const int64_t *offsets, const int64_t *triples) {
    stList *all = stList_construct3(0, (void (*)(void *)) stList_destruct);
    for (int64_t i = 0; i < n; i++) {
        stList *l = stList_construct3(0, (void (*)(void *)) stIntTuple_destruct);
        for (int64_t k = offsets[i]; k < offsets[i + 1]; k++) {
            stList_append(l, stIntTuple_construct3(triples[3 * k], triples[3 * k + 1], triples[3 * k + 2]));
        }
        stList_append(all, l);
    }
    return all;
}

void refpoa_anchors_destroy(void *anchors) {
    stList_destruct(anchors);
}

/* ---- the loop's steps ---- */

void *refpoa_realign(void *reads, void *anchors, const char *refChars, const uint32_t *refCounts, int64_t refLength,
                     void *params) {
    RleString *ref = makeRle(refChars, refCounts, refLength);
    Poa *poa = poa_realign(reads, anchors, ref, params);
    rleString_destruct(ref);
    return poa;
}

void *refpoa_realign_all(void *reads, void *anchors, const char *refChars, const uint32_t *refCounts,
                         int64_t refLength, void *params) {
    RleString *ref = makeRle(refChars, refCounts, refLength);
    Poa *poa = poa_realignAll(reads, anchors, ref, params);
    rleString_destruct(ref);
    return poa;
}

void refpoa_destroy(void *poa) {
    poa_destruct(poa);
}

void refpoa_estimate_repeat_counts(void *poa, void *reads, void *params) {
    poa_estimateRepeatCountsUsingBayesianModel(poa, reads, ((PolishParams *) params)->repeatSubMatrix);
}

double refpoa_score(void *poa) {
    return poa_getReferenceNodeTotalMatchWeight(poa) - poa_getTotalErrorWeight(poa);
}

/* The POA's reference string (chars, counts); returns its run count. */
int64_t refpoa_reference(void *handle, char *chars, uint64_t *counts, int64_t cap) {
    Poa *poa = handle;
    int64_t n = (int64_t) poa->refString->length;
    for (int64_t i = 0; i < n && i < cap; i++) {
        chars[i] = poa->refString->rleString[i];
        counts[i] = poa->refString->repeatCounts[i];
    }
    return n;
}

int64_t refpoa_node_count(void *handle) {
    return stList_length(((Poa *) handle)->nodes);
}

int64_t refpoa_max_repeat(void *handle) {
    return (int64_t) ((Poa *) handle)->maxRepeatCount;
}

/* Node fields: base, repeat count, base weights [n][5], repeat-count weights [n][maxRepeat],
 * and per node the numbers of observations, inserts and deletes. */
void refpoa_nodes(void *handle, char *bases, uint64_t *repeatCounts, double *baseWeights, double *rcWeights,
                  int64_t *nObs, int64_t *nIns, int64_t *nDel) {
    Poa *poa = handle;
    int64_t m = (int64_t) poa->maxRepeatCount;
    for (int64_t i = 0; i < stList_length(poa->nodes); i++) {
        PoaNode *node = stList_get(poa->nodes, i);
        bases[i] = node->base;
        repeatCounts[i] = node->repeatCount;
        for (int64_t k = 0; k < 5; k++) {
            baseWeights[5 * i + k] = node->baseWeights[k];
        }
        for (int64_t k = 0; k < m; k++) {
            rcWeights[m * i + k] = node->repeatCountWeights[k];
        }
        nObs[i] = stList_length(node->observations);
        nIns[i] = stList_length(node->inserts);
        nDel[i] = stList_length(node->deletes);
    }
}

/* Observations of every node in order: (readNo, offset, weight) rows. */
void refpoa_observations(void *handle, int64_t *readNo, int64_t *offset, double *weight) {
    Poa *poa = handle;
    int64_t k = 0;
    for (int64_t i = 0; i < stList_length(poa->nodes); i++) {
        PoaNode *node = stList_get(poa->nodes, i);
        for (int64_t j = 0; j < stList_length(node->observations); j++) {
            PoaBaseObservation *o = stList_get(node->observations, j);
            readNo[k] = o->readNo;
            offset[k] = o->offset;
            weight[k++] = o->weight;
        }
    }
}

/* Inserts of every node in order: weights (forward, reverse), run-length strings laid end
 * to end (lengths[i] runs each), and observation counts. Returns the total run count when
 * chars is NULL. */
int64_t refpoa_inserts(void *handle, double *wF, double *wR, int64_t *lengths, char *chars, uint64_t *counts,
                       int64_t *nObs) {
    Poa *poa = handle;
    int64_t k = 0, runs = 0;
    for (int64_t i = 0; i < stList_length(poa->nodes); i++) {
        PoaNode *node = stList_get(poa->nodes, i);
        for (int64_t j = 0; j < stList_length(node->inserts); j++) {
            PoaInsert *ins = stList_get(node->inserts, j);
            if (chars != NULL) {
                wF[k] = ins->weightForwardStrand;
                wR[k] = ins->weightReverseStrand;
                lengths[k] = (int64_t) ins->insert->length;
                nObs[k] = stList_length(ins->observations);
                for (uint64_t r = 0; r < ins->insert->length; r++) {
                    chars[runs + r] = ins->insert->rleString[r];
                    counts[runs + r] = ins->insert->repeatCounts[r];
                }
            }
            runs += (int64_t) ins->insert->length;
            k++;
        }
    }
    return runs;
}

/* Deletes of every node in order: (length, forward weight, reverse weight, observations). */
void refpoa_deletes(void *handle, int64_t *length, double *wF, double *wR, int64_t *nObs) {
    Poa *poa = handle;
    int64_t k = 0;
    for (int64_t i = 0; i < stList_length(poa->nodes); i++) {
        PoaNode *node = stList_get(poa->nodes, i);
        for (int64_t j = 0; j < stList_length(node->deletes); j++) {
            PoaDelete *del = stList_get(node->deletes, j);
            length[k] = del->length;
            wF[k] = del->weightForwardStrand;
            wR[k] = del->weightReverseStrand;
            nObs[k++] = stList_length(del->observations);
        }
    }
}

/* poa_getConsensus: the consensus run-length string (returns its run count; chars/counts
 * need room for cap runs) and the POA-to-consensus map (node count - 1 entries). */
int64_t refpoa_consensus(void *handle, void *params, char *chars, uint64_t *counts, int64_t cap, int64_t *map) {
    Poa *poa = handle;
    int64_t *m = NULL;
    RleString *c = poa_getConsensus(poa, &m, params);
    int64_t n = (int64_t) c->length;
    for (int64_t i = 0; i < n && i < cap; i++) {
        chars[i] = c->rleString[i];
        counts[i] = c->repeatCounts[i];
    }
    for (int64_t i = 0; i < stList_length(poa->nodes) - 1; i++) {
        map[i] = m[i];
    }
    free(m);
    rleString_destruct(c);
    return n;
}

/* poa_getAnchorAlignments with a given map (NULL: the identity): per read offsets[nReads+1]
 * and triples (consensus position, read offset, expansion); returns the total anchors. */
int64_t refpoa_anchor_alignments(void *handle, const int64_t *map, int64_t nReads, void *params, int64_t *offsets,
                                 int64_t *triples, int64_t cap) {
    stList *a = poa_getAnchorAlignments(handle, (int64_t *) map, nReads, params);
    int64_t k = 0;
    offsets[0] = 0;
    for (int64_t i = 0; i < nReads; i++) {
        stList *l = stList_get(a, i);
        for (int64_t j = 0; j < stList_length(l); j++) {
            stIntTuple *t = stList_get(l, j);
            if (k < cap) {
                triples[3 * k] = stIntTuple_get(t, 0);
                triples[3 * k + 1] = stIntTuple_get(t, 1);
                triples[3 * k + 2] = stIntTuple_get(t, 2);
            }
            k++;
        }
        offsets[i + 1] = k;
    }
    stList_destruct(a);
    return k;
}

/* ---- the polish mode: bubble graph, allele choice, new consensus ---- */

/* bubbleGraph_constructFromPoa (impl/bubbleGraph.c:800-978); sorts the POA's observations
 * in place as the reference does. */
void *refpoa_bubble_graph(void *poa, void *reads, void *params) {
    return bubbleGraph_constructFromPoa(poa, reads, params);
}

void refpoa_bubble_graph_destroy(void *bg) {
    bubbleGraph_destruct(bg);
}

int64_t refpoa_bubble_count(void *handle) {
    return (int64_t) ((BubbleGraph *) handle)->bubbleNo;
}

/* Bubble i: reference start, reference allele length (runs), allele and read counts. */
void refpoa_bubble_info(void *handle, int64_t i, int64_t *refStart, int64_t *refAlleleLength, int64_t *alleleNo,
                        int64_t *readNo) {
    Bubble *b = &((BubbleGraph *) handle)->bubbles[i];
    *refStart = (int64_t) b->refStart;
    *refAlleleLength = (int64_t) b->refAllele->length;
    *alleleNo = (int64_t) b->alleleNo;
    *readNo = (int64_t) b->readNo;
}

/* Allele j of bubble i as a run-length string; returns its run count (copies at most cap). */
int64_t refpoa_bubble_allele(void *handle, int64_t i, int64_t j, char *chars, uint64_t *counts, int64_t cap) {
    RleString *a = ((BubbleGraph *) handle)->bubbles[i].alleles[j];
    for (int64_t k = 0; k < (int64_t) a->length && k < cap; k++) {
        chars[k] = a->rleString[k];
        counts[k] = a->repeatCounts[k];
    }
    return (int64_t) a->length;
}

/* The read substrings of bubble i in the bubble's order: read index in `reads`, start and
 * length in the read's runs, and the mean quality (-1 without qualities). */
void refpoa_bubble_reads(void *handle, int64_t i, void *reads, int64_t *readNo, int64_t *start, int64_t *length,
                         double *qual) {
    Bubble *b = &((BubbleGraph *) handle)->bubbles[i];
    for (int64_t k = 0; k < (int64_t) b->readNo; k++) {
        BamChunkReadSubstring *rs = b->reads[k];
        readNo[k] = -1;
        for (int64_t r = 0; r < stList_length(reads); r++) {
            if (stList_get(reads, r) == rs->read) {
                readNo[k] = r;
                break;
            }
        }
        start[k] = (int64_t) rs->start;
        length[k] = (int64_t) rs->length;
        qual[k] = rs->qualValue;
    }
}

/* The allele supports of bubble i: alleleNo x readNo log-likelihoods (float, allele-major). */
void refpoa_bubble_supports(void *handle, int64_t i, float *out) {
    Bubble *b = &((BubbleGraph *) handle)->bubbles[i];
    memcpy(out, b->alleleReadSupports, sizeof(float) * b->alleleNo * b->readNo);
}

/* bubbleGraph_getConsensusPath then bubbleGraph_getConsensusString: the chosen allele of every
 * bubble (path, bubbleNo entries), the new consensus (returns its run count; copies at most
 * cap runs) and the POA-to-consensus map (reference length entries). */
int64_t refpoa_bubble_consensus(void *handle, void *params, uint64_t *path, char *chars, uint64_t *counts, int64_t cap,
                                int64_t *map) {
    BubbleGraph *bg = handle;
    uint64_t *p = bubbleGraph_getConsensusPath(bg, params);
    memcpy(path, p, sizeof(uint64_t) * bg->bubbleNo);
    int64_t *m = NULL;
    RleString *c = bubbleGraph_getConsensusString(bg, p, &m, params);
    int64_t n = (int64_t) c->length;
    for (int64_t k = 0; k < n && k < cap; k++) {
        chars[k] = c->rleString[k];
        counts[k] = c->repeatCounts[k];
    }
    memcpy(map, m, sizeof(int64_t) * bg->refString->length);
    free(m);
    free(p);
    rleString_destruct(c);
    return n;
}

/* ---- chunk stitching ---- */

/* removeOverlap (impl/polisher.c:1937-2006) on copies of the two strings: returns the overlap
 * match weight and the two crop points. */
int64_t refpoa_remove_overlap(const char *prefix, const char *suffix, int64_t approxOverlap, void *params,
                              int64_t *prefixCropEnd, int64_t *suffixCropStart) {
    char *a = stString_copy(prefix), *b = stString_copy(suffix);
    int64_t w = removeOverlap(a, b, approxOverlap, params, prefixCropEnd, suffixCropStart);
    free(a);
    free(b);
    return w;
}
