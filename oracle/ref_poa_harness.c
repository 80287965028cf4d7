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
 * The bubble-graph polish (poa_polish) is not part of this oracle: its functions, which
 * live in impl/bubbleGraph.c, are stand-ins that abort, and the loop is run with
 * maxRealignmentPolishIterations = 0.
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

/* ---- bubble-graph functions named by impl/polisher.c; never reached in consensus mode ---- */
BubbleGraph *bubbleGraph_constructFromPoa(Poa *poa, stList *bamChunkReads, PolishParams *params) {
    (void) poa, (void) bamChunkReads, (void) params;
    st_errAbort("bubble graph polish is not part of the POA oracle");
    return NULL;
}
void bubbleGraph_destruct(BubbleGraph *bg) {
    (void) bg;
}
uint64_t *bubbleGraph_getConsensusPath(BubbleGraph *bg, PolishParams *polishParams) {
    (void) bg, (void) polishParams;
    st_errAbort("bubble graph polish is not part of the POA oracle");
    return NULL;
}
RleString *bubbleGraph_getConsensusString(BubbleGraph *bg, uint64_t *consensusPath, int64_t **poaToConsensusMap,
                                          PolishParams *polishParams) {
    (void) bg, (void) consensusPath, (void) poaToConsensusMap, (void) polishParams;
    st_errAbort("bubble graph polish is not part of the POA oracle");
    return NULL;
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

static void readDestruct(void *p) {
    BamChunkRead *r = p;
    rleString_destruct(r->rleRead);
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
