/*
 * ref_heap.c — heap blocks of the reference with zeroed slack.  Test
 * infrastructure only (the reference build of oracle/Makefile links it
 * through -Wl,--wrap=malloc,calloc,realloc; nothing in the product does).
 *
 * Why: capture_octahedra_diffuse allocates dc_tmp with gindex + 100 slots
 * when the interface list outgrows it (growth.c:646-660) but indexes the
 * list 1-based (growth.c:666, 779-807), so a step whose list length equals
 * the allocated size writes and reads dc_tmp[size], one decentered_t past
 * the block.  On some decks and decompositions that corrupts the C heap
 * (glibc aborts with "malloc(): memory corruption"; seen on the AM deck
 * split 2 x 2 x 2).  Every block gets 64 extra zeroed bytes, so that slot
 * exists and starts at zero after each (re)allocation, which is the
 * semantics this project's device code gives it.  Nothing else changes:
 * the reference's own sources are compiled unmodified.
 */
#include <stdlib.h>
#include <string.h>

#define SLACK 64

void *__real_malloc(size_t n);
void *__real_calloc(size_t m, size_t n);
void *__real_realloc(void *p, size_t n);

void *__wrap_malloc(size_t n)
{
    char *p = (char *)__real_malloc(n + SLACK);
    if (p) memset(p + n, 0, SLACK);
    return p;
}

void *__wrap_calloc(size_t m, size_t n)
{
    if (n && m > ((size_t)-1 - SLACK) / n) return NULL;
    return __real_calloc(1, m * n + SLACK);
}

void *__wrap_realloc(void *q, size_t n)
{
    char *p = (char *)__real_realloc(q, n + SLACK);
    if (p) memset(p + n, 0, SLACK);
    return p;
}
