/* io.c - the map writers of the reference's example driver (src/io.c),
 * host C.
 *
 * write_rho: the map's doubles, raw and in memory order (src/io.c:89-95).
 *
 * write_image: the map as an 8-bit palette image of log(rho + 1) between the
 * smallest positive and the largest value, scaled to 0..128 as
 * src/io.c:31-47 scales it (zero pixels stay 0); negative or NaN values
 * print a message and write nothing, as src/io.c:15-25 does.  The file is a
 * little-endian baseline TIFF written here without libtiff: one IFD, one
 * uncompressed strip, a 256-entry colour map (the Jet map: red, green and
 * blue each a clamped tent 1.5 - |4x - c| for c = 3, 2, 1 over x = i/255). */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "io.h"

static void put16(unsigned char *p, uint16_t v) {
  p[0] = (unsigned char)(v & 0xff);
  p[1] = (unsigned char)(v >> 8);
}

static void put32(unsigned char *p, uint32_t v) {
  for (int k = 0; k < 4; ++k) p[k] = (unsigned char)(v >> (8 * k));
}

static uint16_t jet(double x, double c) {
  double v = 1.5 - fabs(4.0 * x - c);
  v = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
  return (uint16_t)floor(v * 65535.0 + 0.5);
}

void write_image(char *file_name, double *rho, int grid_dim) {
  if (!file_name || !rho || grid_dim <= 0) return;
  const size_t n = (size_t)grid_dim * grid_dim;
  if ((double)n > 4.0e9) {
    printf("Image too large for a baseline TIFF!\n");
    return;
  }
  for (size_t i = 0; i < n; ++i) {
    if (rho[i] < 0.0) {
      printf("Negative density!\n");
      return;
    }
    if (rho[i] != rho[i]) {
      printf("Nan density!\n");
      return;
    }
  }
  double max_val = 0.0, min_val = INFINITY;
  for (size_t i = 0; i < n; ++i) {
    if (rho[i] > max_val) max_val = rho[i];
    if (rho[i] > 0.0 && rho[i] < min_val) min_val = rho[i];
  }
  unsigned char *image = (unsigned char *)malloc(n);
  if (!image) return;
  const double lo = log(min_val + 1.0), span = log(max_val + 1.0) - lo;
  for (size_t i = 0; i < n; ++i)
    image[i] = (rho[i] > 0.0 && span > 0.0) ? (unsigned char)(128.0 * (log(rho[i] + 1.0) - lo) / span)
                                            : 0;

  enum { kEntries = 12 };
  const uint32_t ifd = 8, ifd_bytes = 2 + 12 * kEntries + 4;
  const uint32_t cmap = ifd + ifd_bytes, data = cmap + 3 * 256 * 2;
  unsigned char head[8 + 2 + 12 * kEntries + 4 + 3 * 256 * 2];
  memset(head, 0, sizeof(head));
  head[0] = 'I';
  head[1] = 'I';
  put16(head + 2, 42);
  put32(head + 4, ifd);
  unsigned char *e = head + ifd;
  put16(e, kEntries);
  e += 2;
  /* tag, type (3 SHORT, 4 LONG), count, value or offset; ascending tags */
  const uint32_t entries[kEntries][4] = {
      {256, 4, 1, (uint32_t)grid_dim},       /* ImageWidth */
      {257, 4, 1, (uint32_t)grid_dim},       /* ImageLength */
      {258, 3, 1, 8},                        /* BitsPerSample */
      {259, 3, 1, 1},                        /* Compression: none */
      {262, 3, 1, 3},                        /* PhotometricInterpretation: palette */
      {273, 4, 1, data},                     /* StripOffsets */
      {274, 3, 1, 1},                        /* Orientation: top left */
      {277, 3, 1, 1},                        /* SamplesPerPixel */
      {278, 4, 1, (uint32_t)grid_dim},       /* RowsPerStrip: one strip */
      {279, 4, 1, (uint32_t)n},              /* StripByteCounts */
      {284, 3, 1, 1},                        /* PlanarConfiguration: contiguous */
      {320, 3, 3 * 256, cmap},               /* ColorMap */
  };
  for (int k = 0; k < kEntries; ++k, e += 12) {
    put16(e, (uint16_t)entries[k][0]);
    put16(e + 2, (uint16_t)entries[k][1]);
    put32(e + 4, entries[k][2]);
    if (entries[k][1] == 3 && entries[k][2] == 1) put16(e + 8, (uint16_t)entries[k][3]);
    else put32(e + 8, entries[k][3]);
  }
  put32(e, 0); /* no further IFD */
  for (int i = 0; i < 256; ++i) {
    const double x = i / 255.0;
    put16(head + cmap + 2 * i, jet(x, 3.0));
    put16(head + cmap + 2 * (256 + i), jet(x, 2.0));
    put16(head + cmap + 2 * (512 + i), jet(x, 1.0));
  }
  FILE *f = fopen(file_name, "wb");
  if (!f) {
    fprintf(stderr, "write_image: cannot open %s\n", file_name);
    free(image);
    return;
  }
  if (fwrite(head, 1, sizeof(head), f) != sizeof(head) || fwrite(image, 1, n, f) != n)
    fprintf(stderr, "write_image: short write to %s\n", file_name);
  fclose(f);
  free(image);
}

int write_rho(char *fname, double **rho, int rho_size) {
  if (!fname || !rho || !*rho || rho_size < 0) return 0;
  FILE *outfile = fopen(fname, "wb");
  if (!outfile) {
    fprintf(stderr, "write_rho: cannot open %s\n", fname);
    return 0;
  }
  const int written = (int)fwrite(*rho, sizeof(double), (size_t)rho_size, outfile);
  fclose(outfile);
  return written;
}
