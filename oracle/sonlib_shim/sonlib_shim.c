/*
 * Project-written implementation of the small sonLib API surface declared in
 * include/sonLib.h. TEST INFRASTRUCTURE ONLY: it lets the reference's
 * impl/pairwiseAligner.c and impl/stateMachine.c be compiled unmodified as an
 * oracle, and it stands in for the host application's sonLib when the drop-in
 * library is exercised by the tests.
 *
 * Semantics follow the way the reference uses each call:
 *  - stList is a growable pointer array; stList_pop removes the last element
 *    (impl/pairwiseAligner.c:1072-1074 relies on that to reverse sub-lists);
 *  - stIntTuple is int64_t[1 + n] with the length in slot 0 (impl/polisher.c:597);
 *  - stThrowNew is only reached on invalid diagonals (impl/pairwiseAligner.c:23-27),
 *    a bug path, so it aborts with the message.
 */
#include "sonLib.h"

/* ---------------- memory ---------------- */

void *st_malloc(int64_t size) {
    void *p = malloc(size > 0 ? (size_t) size : 1);
    if (p == NULL) {
        fprintf(stderr, "sonlib_shim: out of memory (%" PRIi64 " bytes)\n", size);
        abort();
    }
    return p;
}

void *st_calloc(int64_t elementNumber, int64_t elementSize) {
    void *p = calloc(elementNumber > 0 ? (size_t) elementNumber : 1, elementSize > 0 ? (size_t) elementSize : 1);
    if (p == NULL) {
        fprintf(stderr, "sonlib_shim: out of memory\n");
        abort();
    }
    return p;
}

/* ---------------- errors and logging ---------------- */

static int shimLogLevel = 0; /* 0 = quiet */

void st_errAbort(const char *msg, ...) {
    va_list ap;
    va_start(ap, msg);
    vfprintf(stderr, msg, ap);
    va_end(ap);
    fputc('\n', stderr);
    exit(1);
}

void stThrowNew(const char *id, const char *msg, ...) {
    va_list ap;
    fprintf(stderr, "%s: ", id);
    va_start(ap, msg);
    vfprintf(stderr, msg, ap);
    va_end(ap);
    fputc('\n', stderr);
    abort();
}

static void shimLog(int level, const char *msg, va_list ap) {
    if (shimLogLevel >= level) {
        vfprintf(stderr, msg, ap);
    }
}

void st_logDebug(const char *msg, ...) {
    va_list ap;
    va_start(ap, msg);
    shimLog(3, msg, ap);
    va_end(ap);
}

void st_logInfo(const char *msg, ...) {
    va_list ap;
    va_start(ap, msg);
    shimLog(2, msg, ap);
    va_end(ap);
}

void st_logCritical(const char *msg, ...) {
    va_list ap;
    va_start(ap, msg);
    shimLog(1, msg, ap);
    va_end(ap);
}

int st_getLogLevel(void) {
    return shimLogLevel;
}

/* ---------------- strings ---------------- */

char *stString_print(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    int n = vsnprintf(NULL, 0, fmt, ap);
    va_end(ap);
    char *s = st_malloc(n + 1);
    va_start(ap, fmt);
    vsnprintf(s, n + 1, fmt, ap);
    va_end(ap);
    return s;
}

char *stString_copy(const char *s) {
    size_t n = strlen(s);
    char *c = st_malloc(n + 1);
    memcpy(c, s, n + 1);
    return c;
}

bool stString_eq(const char *a, const char *b) {
    if (a == NULL || b == NULL) {
        return a == b;
    }
    return strcmp(a, b) == 0;
}

/* ---------------- random numbers: splitmix64, seedable ---------------- */

static uint64_t shimRngState = 0x853c49e6748fea9bULL;

void st_randomSeed(uint64_t seed) {
    shimRngState = seed;
}

static uint64_t shimNext(void) {
    uint64_t z = (shimRngState += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

double st_random(void) {
    return (double) (shimNext() >> 11) * (1.0 / 9007199254740992.0);
}

/* Uniform integer in [min, max). */
int64_t st_randomInt(int64_t min, int64_t max) {
    if (max <= min) {
        st_errAbort("st_randomInt: empty range [%" PRIi64 ", %" PRIi64 ")", min, max);
    }
    return min + (int64_t) (shimNext() % (uint64_t) (max - min));
}

/* ---------------- stList ---------------- */

struct _stList {
    void **items;
    int64_t length;
    int64_t capacity;
    void (*destructElement)(void *);
};

stList *stList_construct3(int64_t length, void (*destructElement)(void *)) {
    stList *l = st_malloc(sizeof(stList));
    l->capacity = length > 4 ? length : 4;
    l->items = st_calloc(l->capacity, sizeof(void *));
    l->length = length;
    l->destructElement = destructElement;
    return l;
}

stList *stList_construct2(int64_t length) {
    return stList_construct3(length, NULL);
}

stList *stList_construct(void) {
    return stList_construct3(0, NULL);
}

void stList_setDestructor(stList *list, void (*destructElement)(void *)) {
    list->destructElement = destructElement;
}

void stList_destruct(stList *list) {
    if (list == NULL) {
        return;
    }
    if (list->destructElement != NULL) {
        for (int64_t i = 0; i < list->length; i++) {
            if (list->items[i] != NULL) {
                list->destructElement(list->items[i]);
            }
        }
    }
    free(list->items);
    free(list);
}

void stList_append(stList *list, void *item) {
    if (list->length == list->capacity) {
        list->capacity *= 2;
        list->items = realloc(list->items, sizeof(void *) * list->capacity);
        if (list->items == NULL) {
            st_errAbort("sonlib_shim: out of memory in stList_append");
        }
    }
    list->items[list->length++] = item;
}

void *stList_get(stList *list, int64_t index) {
    if (index < 0 || index >= list->length) {
        st_errAbort("stList_get: index %" PRIi64 " out of range (length %" PRIi64 ")", index, list->length);
    }
    return list->items[index];
}

void stList_set(stList *list, int64_t index, void *item) {
    if (index < 0 || index >= list->length) {
        st_errAbort("stList_set: index %" PRIi64 " out of range", index);
    }
    list->items[index] = item;
}

int64_t stList_length(stList *list) {
    return list->length;
}

void *stList_peek(stList *list) {
    if (list->length == 0) {
        st_errAbort("stList_peek: empty list");
    }
    return list->items[list->length - 1];
}

void *stList_pop(stList *list) {
    if (list->length == 0) {
        st_errAbort("stList_pop: empty list");
    }
    return list->items[--list->length];
}

void stList_reverse(stList *list) {
    for (int64_t i = 0, j = list->length - 1; i < j; i++, j--) {
        void *t = list->items[i];
        list->items[i] = list->items[j];
        list->items[j] = t;
    }
}

/* ---------------- stIntTuple ---------------- */

static stIntTuple *tupleAlloc(int64_t n) {
    stIntTuple *t = st_malloc(sizeof(int64_t) * (n + 1));
    t[0] = n;
    return t;
}

stIntTuple *stIntTuple_construct1(int64_t v1) {
    stIntTuple *t = tupleAlloc(1);
    t[1] = v1;
    return t;
}

stIntTuple *stIntTuple_construct2(int64_t v1, int64_t v2) {
    stIntTuple *t = tupleAlloc(2);
    t[1] = v1;
    t[2] = v2;
    return t;
}

stIntTuple *stIntTuple_construct3(int64_t v1, int64_t v2, int64_t v3) {
    stIntTuple *t = tupleAlloc(3);
    t[1] = v1;
    t[2] = v2;
    t[3] = v3;
    return t;
}

stIntTuple *stIntTuple_construct4(int64_t v1, int64_t v2, int64_t v3, int64_t v4) {
    stIntTuple *t = tupleAlloc(4);
    t[1] = v1;
    t[2] = v2;
    t[3] = v3;
    t[4] = v4;
    return t;
}

void stIntTuple_destruct(stIntTuple *t) {
    free(t);
}

int64_t stIntTuple_get(stIntTuple *t, int64_t index) {
    if (index < 0 || index >= t[0]) {
        st_errAbort("stIntTuple_get: index %" PRIi64 " out of range", index);
    }
    return t[index + 1];
}

int64_t stIntTuple_length(stIntTuple *t) {
    return t[0];
}

int stIntTuple_cmpFn(stIntTuple *a, stIntTuple *b) {
    int64_t n = a[0] < b[0] ? a[0] : b[0];
    for (int64_t i = 1; i <= n; i++) {
        if (a[i] != b[i]) {
            return a[i] < b[i] ? -1 : 1;
        }
    }
    return a[0] == b[0] ? 0 : (a[0] < b[0] ? -1 : 1);
}

int stIntTuple_equalsFn(stIntTuple *a, stIntTuple *b) {
    return stIntTuple_cmpFn(a, b) == 0;
}

/* ---------------- JSON: unused by the oracle, so these stop loudly ---------------- */

int64_t stJson_setupParser(char *buf, size_t r, jsmntok_t **tokens, char **js) {
    (void) buf; (void) r; (void) tokens; (void) js;
    st_errAbort("sonlib_shim: JSON parsing is not provided; fill parameters directly");
    return 0;
}

char *stJson_token_tostr(char *js, jsmntok_t *t) {
    (void) js; (void) t;
    st_errAbort("sonlib_shim: JSON parsing is not provided");
    return NULL;
}

int64_t stJson_parseInt(char *js, jsmntok_t *tokens, int64_t tokenIndex) {
    (void) js; (void) tokens; (void) tokenIndex;
    st_errAbort("sonlib_shim: JSON parsing is not provided");
    return 0;
}

double stJson_parseFloat(char *js, jsmntok_t *tokens, int64_t tokenIndex) {
    (void) js; (void) tokens; (void) tokenIndex;
    st_errAbort("sonlib_shim: JSON parsing is not provided");
    return 0.0;
}

bool stJson_parseBool(char *js, jsmntok_t *tokens, int64_t tokenIndex) {
    (void) js; (void) tokens; (void) tokenIndex;
    st_errAbort("sonlib_shim: JSON parsing is not provided");
    return 0;
}

int64_t stJson_parseFloatArray(double *array, int64_t length, char *js, jsmntok_t *tokens, int64_t tokenIndex) {
    (void) array; (void) length; (void) js; (void) tokens; (void) tokenIndex;
    st_errAbort("sonlib_shim: JSON parsing is not provided");
    return 0;
}
