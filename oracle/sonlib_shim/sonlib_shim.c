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

/* ---------------- stList_sort ---------------- */

/* qsort hands the comparator pointers to the array slots; sonLib's comparators take the
 * list items themselves. */
static __thread int (*gListCmp)(const void *, const void *);

static int listSlotCmp(const void *a, const void *b) {
    return gListCmp(*(void *const *) a, *(void *const *) b);
}

void stList_sort(stList *list, int (*cmpFn)(const void *a, const void *b)) {
    int (*saved)(const void *, const void *) = gListCmp;
    gListCmp = cmpFn;
    qsort(list->items, (size_t) list->length, sizeof(void *), listSlotCmp);
    gListCmp = saved;
}

/* ---------------- stSortedSet ---------------- */

struct _stSortedSet {
    void **items;
    int64_t length, capacity;
    int (*cmp)(const void *, const void *);
    void (*destructElement)(void *);
};

stSortedSet *stSortedSet_construct3(int (*cmpFn)(const void *, const void *), void (*destructElementFn)(void *)) {
    stSortedSet *s = st_calloc(1, sizeof(stSortedSet));
    s->capacity = 16;
    s->items = st_calloc(s->capacity, sizeof(void *));
    s->cmp = cmpFn;
    s->destructElement = destructElementFn;
    return s;
}

void stSortedSet_destruct(stSortedSet *set) {
    if (set == NULL) {
        return;
    }
    if (set->destructElement != NULL) {
        for (int64_t i = 0; i < set->length; i++) {
            set->destructElement(set->items[i]);
        }
    }
    free(set->items);
    free(set);
}

/* first index whose item is not less than object */
static int64_t sortedLowerBound(stSortedSet *set, void *object) {
    int64_t lo = 0, hi = set->length;
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (set->cmp(set->items[mid], object) < 0) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo;
}

void stSortedSet_insert(stSortedSet *set, void *object) {
    int64_t i = sortedLowerBound(set, object);
    if (i < set->length && set->cmp(set->items[i], object) == 0) { /* a set: replace the equal item */
        set->items[i] = object;
        return;
    }
    if (set->length == set->capacity) {
        set->capacity *= 2;
        set->items = realloc(set->items, sizeof(void *) * set->capacity);
    }
    memmove(set->items + i + 1, set->items + i, sizeof(void *) * (set->length - i));
    set->items[i] = object;
    set->length++;
}

void *stSortedSet_search(stSortedSet *set, void *object) {
    int64_t i = sortedLowerBound(set, object);
    return (i < set->length && set->cmp(set->items[i], object) == 0) ? set->items[i] : NULL;
}

/* ---------------- stHash (linear probing; insertion-ordered iteration) ----------------
 * Keys hash by pointer value unless construct3 gives a hash and an equality function.
 * Every key also sits in `order` (insertion order, removed keys taken out), which is
 * the order the iterator visits. */

struct _stHash {
    void **keys;
    void **values;
    char *used;
    int64_t size, count;
    uint64_t (*hashKey)(const void *);
    int (*equalKeys)(const void *, const void *);
    void (*destructKeys)(void *);
    void (*destructValues)(void *);
    void **order;
    int64_t orderLength, orderCap;
};

struct _stHashIterator {
    stHash *hash;
    int64_t next;
};

static stHash *hashAlloc(void) {
    stHash *h = st_calloc(1, sizeof(stHash));
    h->size = 64;
    h->keys = st_calloc(h->size, sizeof(void *));
    h->values = st_calloc(h->size, sizeof(void *));
    h->used = st_calloc(h->size, 1);
    return h;
}

stHash *stHash_construct(void) {
    return hashAlloc();
}

stHash *stHash_construct2(void (*destructKeys)(void *), void (*destructValues)(void *)) {
    stHash *h = hashAlloc();
    h->destructKeys = destructKeys;
    h->destructValues = destructValues;
    return h;
}

stHash *stHash_construct3(uint64_t (*hashKey)(const void *), int (*hashEqualsKey)(const void *, const void *),
                          void (*destructKeys)(void *), void (*destructValues)(void *)) {
    stHash *h = stHash_construct2(destructKeys, destructValues);
    h->hashKey = hashKey;
    h->equalKeys = hashEqualsKey;
    return h;
}

void stHash_destruct(stHash *hash) {
    if (hash == NULL) {
        return;
    }
    for (int64_t i = 0; i < hash->size; i++) {
        if (hash->used[i]) {
            if (hash->destructKeys != NULL) {
                hash->destructKeys(hash->keys[i]);
            }
            if (hash->destructValues != NULL) {
                hash->destructValues(hash->values[i]);
            }
        }
    }
    free(hash->keys);
    free(hash->values);
    free(hash->used);
    free(hash->order);
    free(hash);
}

static int sameKey(stHash *h, void *a, void *b) {
    return h->equalKeys != NULL ? h->equalKeys(a, b) != 0 : a == b;
}

static int64_t hashSlot(stHash *h, void *key) {
    uint64_t x = h->hashKey != NULL ? h->hashKey(key) : (uint64_t) (uintptr_t) key;
    x *= 0x9E3779B97F4A7C15ull;
    int64_t i = (int64_t) (x >> 17) & (h->size - 1);
    while (h->used[i] && !sameKey(h, h->keys[i], key)) {
        i = (i + 1) & (h->size - 1);
    }
    return i;
}

/* places a key that is not in the table (no order bookkeeping) */
static void hashPlace(stHash *hash, void *key, void *value) {
    int64_t i = hashSlot(hash, key);
    hash->used[i] = 1;
    hash->keys[i] = key;
    hash->values[i] = value;
    hash->count++;
}

void stHash_insert(stHash *hash, void *key, void *value) {
    int64_t i = hashSlot(hash, key);
    if (hash->used[i]) {
        hash->values[i] = value;
        return;
    }
    if (2 * (hash->count + 1) > hash->size) {
        stHash old = *hash;
        hash->size *= 2;
        hash->count = 0;
        hash->keys = st_calloc(hash->size, sizeof(void *));
        hash->values = st_calloc(hash->size, sizeof(void *));
        hash->used = st_calloc(hash->size, 1);
        for (int64_t k = 0; k < old.size; k++) {
            if (old.used[k]) {
                hashPlace(hash, old.keys[k], old.values[k]);
            }
        }
        free(old.keys);
        free(old.values);
        free(old.used);
    }
    hashPlace(hash, key, value);
    if (hash->orderLength == hash->orderCap) {
        hash->orderCap = hash->orderCap ? 2 * hash->orderCap : 16;
        hash->order = realloc(hash->order, sizeof(void *) * (size_t) hash->orderCap);
        if (hash->order == NULL) {
            st_errAbort("stHash: out of memory");
        }
    }
    hash->order[hash->orderLength++] = key;
}

void *stHash_search(stHash *hash, void *key) {
    int64_t i = hashSlot(hash, key);
    return hash->used[i] ? hash->values[i] : NULL;
}

void *stHash_remove(stHash *hash, void *key) {
    int64_t i = hashSlot(hash, key);
    if (!hash->used[i]) {
        return NULL;
    }
    void *v = hash->values[i];
    void *stored = hash->keys[i];
    for (int64_t k = 0; k < hash->orderLength; k++) {
        if (hash->order[k] == stored) {
            memmove(hash->order + k, hash->order + k + 1, sizeof(void *) * (size_t) (hash->orderLength - k - 1));
            hash->orderLength--;
            break;
        }
    }
    /* re-place the rest of the probe run */
    hash->used[i] = 0;
    hash->count--;
    int64_t j = (i + 1) & (hash->size - 1);
    while (hash->used[j]) {
        void *k = hash->keys[j], *val = hash->values[j];
        hash->used[j] = 0;
        hash->count--;
        hashPlace(hash, k, val);
        j = (j + 1) & (hash->size - 1);
    }
    return v;
}

stHashIterator *stHash_getIterator(stHash *hash) {
    stHashIterator *it = st_calloc(1, sizeof(stHashIterator));
    it->hash = hash;
    return it;
}

void *stHash_getNext(stHashIterator *iterator) {
    return iterator->next < iterator->hash->orderLength ? iterator->hash->order[iterator->next++] : NULL;
}

void stHash_destructIterator(stHashIterator *iterator) {
    free(iterator);
}

stList *stHash_getValues(stHash *hash) {
    stList *l = stList_construct();
    for (int64_t k = 0; k < hash->orderLength; k++) {
        stList_append(l, stHash_search(hash, hash->order[k]));
    }
    return l;
}

/* FNV-1a over the string's bytes */
uint64_t stHash_stringKey(const char *k) {
    uint64_t h = 1469598103934665603ull;
    for (const unsigned char *c = (const unsigned char *) k; *c; c++) {
        h = (h ^ *c) * 1099511628211ull;
    }
    return h;
}

/* ---------------- stSet, stMath_logAddExact: phasing only ---------------- */

#define PHASING_ONLY(name) st_errAbort("%s: phasing is not part of the oracle", name)

stSet *stSet_construct(void) {
    PHASING_ONLY("stSet_construct");
    return NULL;
}
void stSet_destruct(stSet *set) {
    (void) set;
    PHASING_ONLY("stSet_destruct");
}
void stSet_insert(stSet *set, void *object) {
    (void) set, (void) object;
    PHASING_ONLY("stSet_insert");
}
void *stSet_search(stSet *set, void *object) {
    (void) set, (void) object;
    PHASING_ONLY("stSet_search");
    return NULL;
}
int64_t stSet_size(stSet *set) {
    (void) set;
    PHASING_ONLY("stSet_size");
    return 0;
}
stSet *stSet_getIntersection(stSet *set1, stSet *set2) {
    (void) set1, (void) set2;
    PHASING_ONLY("stSet_getIntersection");
    return NULL;
}
stSetIterator *stSet_getIterator(stSet *set) {
    (void) set;
    PHASING_ONLY("stSet_getIterator");
    return NULL;
}
void *stSet_getNext(stSetIterator *iterator) {
    (void) iterator;
    PHASING_ONLY("stSet_getNext");
    return NULL;
}
void stSet_destructIterator(stSetIterator *iterator) {
    (void) iterator;
    PHASING_ONLY("stSet_destructIterator");
}
stSet *stList_getSet(stList *list) {
    (void) list;
    PHASING_ONLY("stList_getSet");
    return NULL;
}
double stMath_logAddExact(double logX, double logY) {
    (void) logX, (void) logY;
    PHASING_ONLY("stMath_logAddExact");
    return 0.0;
}

/* ---------------- strings ---------------- */

char *stString_getSubString(const char *cA, int64_t start, int64_t length) {
    char *c = st_malloc(length + 1);
    memcpy(c, cA + start, (size_t) length);
    c[length] = '\0';
    return c;
}

char *stString_join2(const char *pad, stList *strings) {
    size_t padLen = strlen(pad), total = 1;
    for (int64_t i = 0; i < strings->length; i++) {
        total += strlen(strings->items[i]) + (i > 0 ? padLen : 0);
    }
    char *out = st_malloc((int64_t) total);
    size_t k = 0;
    for (int64_t i = 0; i < strings->length; i++) {
        if (i > 0) {
            memcpy(out + k, pad, padLen);
            k += padLen;
        }
        size_t n = strlen(strings->items[i]);
        memcpy(out + k, strings->items[i], n);
        k += n;
    }
    out[k] = '\0';
    return out;
}
