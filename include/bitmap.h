/*
 * bitmap.h - the face bitmap passed between find_forward_hull and
 * copy_fh_triangles.  Replaces src/bitmap.h:1-19 of the reference.
 *
 * Layout kept for ABI compatibility: the reference stores
 * sizeof(word_t)*sizeof(char) = 4 bits per 32-bit word (src/bitmap.c:8), so
 * bit 4*t+f (face f of tet t) lives in word t, bit f.  create_bitmap(n)
 * allocates n/4 + 1 zeroed words with calloc; free it with delete_bitmap or
 * free().
 */
#ifndef SDTFE_BITMAP_H
#define SDTFE_BITMAP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef uint32_t word_t;

void set_bit(word_t *words, int n);      /* src/bitmap.c:13-15 */
void clear_bit(word_t *words, int n);    /* src/bitmap.c:17-19 */
int get_bit(word_t *words, int n);       /* src/bitmap.c:21-24 */
word_t *create_bitmap(int n);            /* src/bitmap.c:26-28 */
void delete_bitmap(word_t *words);       /* src/bitmap.c:30-32 */

#ifdef __cplusplus
}
#endif
#endif
