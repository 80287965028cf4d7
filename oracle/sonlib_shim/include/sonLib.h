/*
 * Minimal stand-in for the sonLib API surface used by MarginPolish's pair-HMM
 * sources (impl/pairwiseAligner.c, impl/stateMachine.c) and by the POA loop of
 * impl/polisher.c.
 *
 * TEST INFRASTRUCTURE ONLY. sonLib (a git submodule of the reference) is not
 * present, so this header declares, from the way the reference calls them, the
 * containers, allocation, logging and error helpers those two files use. The
 * implementation is sonlib_shim.c, written for this project. Only the oracle
 * build (oracle/Makefile) and the drop-in test host use it.
 *
 * Layout note: stIntTuple is an int64_t array whose element 0 holds the tuple
 * length and whose values start at element 1. impl/polisher.c:597 and
 * :169-175 poke tuples through that layout directly, so it is kept.
 */
#ifndef MP_SONLIB_SHIM_H_
#define MP_SONLIB_SHIM_H_

#include <assert.h>
#include <stdint.h>
#include <stdlib.h>
#include <stdio.h>
#include <stdbool.h>
#include <stdarg.h>
#include <string.h>
#include <math.h>
#include <inttypes.h>
#include <limits.h>

#ifndef TRUE
#define TRUE 1
#endif
#ifndef FALSE
#define FALSE 0
#endif

#define LOG_ONE 0.0

#ifdef __cplusplus
extern "C" {
#endif

/* opaque container types named by the reference headers */
typedef struct _stList stList;
typedef int64_t stIntTuple;
typedef struct _stSet stSet;
typedef struct _stHash stHash;
typedef struct _stSortedSet stSortedSet;
typedef struct _stListIterator stListIterator;
typedef struct _stSetIterator stSetIterator;
typedef struct _stHashIterator stHashIterator;
typedef struct _stSortedSetIterator stSortedSetIterator;

/* jsmn token type: only named in prototypes of the two hot-path files */
typedef struct {
    int type;
    int start;
    int end;
    int size;
} jsmntok_t;

/* ---- memory ---- */
void *st_malloc(int64_t size);
void *st_calloc(int64_t elementNumber, int64_t elementSize);

/* ---- errors and logging ---- */
void st_errAbort(const char *msg, ...);
void stThrowNew(const char *id, const char *msg, ...);
void st_logDebug(const char *msg, ...);
void st_logInfo(const char *msg, ...);
void st_logCritical(const char *msg, ...);
int st_getLogLevel(void);
/* log levels compared against st_getLogLevel() (impl/polisher.c:1974) */
enum stLogLevel { off = 0, critical = 1, info = 2, debug = 3 };

/* ---- strings ---- */
char *stString_print(const char *fmt, ...);
char *stString_copy(const char *s);
bool stString_eq(const char *a, const char *b);

/* ---- random numbers (seedable) ---- */
void st_randomSeed(uint64_t seed);
double st_random(void);
int64_t st_randomInt(int64_t min, int64_t max);

/* ---- stList ---- */
stList *stList_construct(void);
stList *stList_construct2(int64_t length);
stList *stList_construct3(int64_t length, void (*destructElement)(void *));
void stList_destruct(stList *list);
void stList_append(stList *list, void *item);
void *stList_get(stList *list, int64_t index);
void stList_set(stList *list, int64_t index, void *item);
int64_t stList_length(stList *list);
void *stList_peek(stList *list);
void *stList_pop(stList *list);
void stList_reverse(stList *list);
void stList_setDestructor(stList *list, void (*destructElement)(void *));

void stList_sort(stList *list, int (*cmpFn)(const void *a, const void *b));

/* ---- stSortedSet (a sorted array; the POA oracle's match sets) ---- */
stSortedSet *stSortedSet_construct3(int (*cmpFn)(const void *, const void *), void (*destructElementFn)(void *));
void stSortedSet_destruct(stSortedSet *set);
void stSortedSet_insert(stSortedSet *set, void *object);
void *stSortedSet_search(stSortedSet *set, void *object);

/* ---- stHash: keyed by pointer value, or by the caller's hash and equality functions
 * (construct3, as impl/bubbleGraph.c:728 and :905 use it). Iteration visits the keys in
 * insertion order; sonLib's own table visits them in bucket order, which only decides
 * the order of equal-likelihood alleles in the bubble graph. ---- */
stHash *stHash_construct(void);
stHash *stHash_construct2(void (*destructKeys)(void *), void (*destructValues)(void *));
stHash *stHash_construct3(uint64_t (*hashKey)(const void *), int (*hashEqualsKey)(const void *, const void *),
                          void (*destructKeys)(void *), void (*destructValues)(void *));
void stHash_destruct(stHash *hash);
void stHash_insert(stHash *hash, void *key, void *value);
void *stHash_search(stHash *hash, void *key);
void *stHash_remove(stHash *hash, void *key);
stHashIterator *stHash_getIterator(stHash *hash);
void *stHash_getNext(stHashIterator *iterator);
void stHash_destructIterator(stHashIterator *iterator);
stList *stHash_getValues(stHash *hash);
uint64_t stHash_stringKey(const char *k);

/* ---- stSet and stMath_logAddExact: named by the phasing code of impl/bubbleGraph.c, which
 * the oracle never runs (they abort) ---- */
stSet *stSet_construct(void);
void stSet_destruct(stSet *set);
void stSet_insert(stSet *set, void *object);
void *stSet_search(stSet *set, void *object);
int64_t stSet_size(stSet *set);
stSet *stSet_getIntersection(stSet *set1, stSet *set2);
stSetIterator *stSet_getIterator(stSet *set);
void *stSet_getNext(stSetIterator *iterator);
void stSet_destructIterator(stSetIterator *iterator);
stSet *stList_getSet(stList *list);
double stMath_logAddExact(double logX, double logY);

/* ---- more strings ---- */
char *stString_getSubString(const char *cA, int64_t start, int64_t length);
char *stString_join2(const char *pad, stList *strings);

/* ---- stIntTuple ---- */
stIntTuple *stIntTuple_construct1(int64_t v1);
stIntTuple *stIntTuple_construct2(int64_t v1, int64_t v2);
stIntTuple *stIntTuple_construct3(int64_t v1, int64_t v2, int64_t v3);
stIntTuple *stIntTuple_construct4(int64_t v1, int64_t v2, int64_t v3, int64_t v4);
void stIntTuple_destruct(stIntTuple *t);
int64_t stIntTuple_get(stIntTuple *t, int64_t index);
int64_t stIntTuple_length(stIntTuple *t);
int stIntTuple_cmpFn(stIntTuple *a, stIntTuple *b);
int stIntTuple_equalsFn(stIntTuple *a, stIntTuple *b);

/* ---- JSON (not used by the oracle harness; parameters are filled directly) ---- */
int64_t stJson_setupParser(char *buf, size_t r, jsmntok_t **tokens, char **js);
char *stJson_token_tostr(char *js, jsmntok_t *t);
int64_t stJson_parseInt(char *js, jsmntok_t *tokens, int64_t tokenIndex);
double stJson_parseFloat(char *js, jsmntok_t *tokens, int64_t tokenIndex);
bool stJson_parseBool(char *js, jsmntok_t *tokens, int64_t tokenIndex);
int64_t stJson_parseFloatArray(double *array, int64_t length, char *js, jsmntok_t *tokens, int64_t tokenIndex);

#ifdef __cplusplus
}
#endif

#endif
