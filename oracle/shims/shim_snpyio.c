/*
 * NPY header reader/writer (see snpyio.h).  TEST INFRASTRUCTURE ONLY.
 * Format: magic "\x93NUMPY", major, minor, little-endian header length
 * (2 bytes for v1, 4 bytes for v2), then a Python dict literal padded with
 * spaces and a final '\n' so that the data starts on a 64-byte boundary.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "snpyio.h"

static const char *skip_ws(const char *s) {
  while (*s == ' ') s++;
  return s;
}

int snpyio_r_header(size_t *ndim, size_t **shape, char **dtype, bool *is_fortran_order,
                    FILE *fp, size_t *header_size) {
  unsigned char pre[10];
  if (8 != fread(pre, 1, 8, fp)) return 1;
  if (pre[0] != 0x93 || 0 != memcmp(pre + 1, "NUMPY", 5)) return 1;
  size_t hlen = 0, prelen = 0;
  if (1 == pre[6]) {
    unsigned char b[2];
    if (2 != fread(b, 1, 2, fp)) return 1;
    hlen = (size_t)b[0] | ((size_t)b[1] << 8);
    prelen = 10;
  } else if (2 == pre[6] || 3 == pre[6]) {
    unsigned char b[4];
    if (4 != fread(b, 1, 4, fp)) return 1;
    hlen = (size_t)b[0] | ((size_t)b[1] << 8) | ((size_t)b[2] << 16) | ((size_t)b[3] << 24);
    prelen = 12;
  } else {
    return 1;
  }
  char *dict = calloc(hlen + 1, 1);
  if (hlen != fread(dict, 1, hlen, fp)) { free(dict); return 1; }
  /* descr */
  const char *d = strstr(dict, "'descr'");
  const char *f = strstr(dict, "'fortran_order'");
  const char *s = strstr(dict, "'shape'");
  if (!d || !f || !s) { free(dict); return 1; }
  d = strchr(d + 7, ':');
  if (!d) { free(dict); return 1; }
  d = skip_ws(d + 1);
  if (*d != '\'') { free(dict); return 1; }
  const char *e = strchr(d + 1, '\'');
  if (!e) { free(dict); return 1; }
  const size_t dlen = (size_t)(e - d) + 1;
  *dtype = calloc(dlen + 1, 1);
  memcpy(*dtype, d, dlen);
  /* fortran_order */
  f = strchr(f + 15, ':');
  f = skip_ws(f + 1);
  *is_fortran_order = (0 == strncmp(f, "True", 4));
  /* shape */
  s = strchr(s + 7, '(');
  if (!s) { free(dict); free(*dtype); return 1; }
  s++;
  size_t cap = 8, n = 0;
  size_t *sh = calloc(cap, sizeof(size_t));
  while (1) {
    s = skip_ws(s);
    if (*s == ')') break;
    char *end = NULL;
    const unsigned long long v = strtoull(s, &end, 10);
    if (end == s) { free(sh); free(dict); free(*dtype); return 1; }
    if (n == cap) { cap *= 2; sh = realloc(sh, cap * sizeof(size_t)); }
    sh[n++] = (size_t)v;
    s = skip_ws(end);
    if (*s == ',') s++;
  }
  *ndim = n;
  *shape = sh;
  *header_size = prelen + hlen;
  free(dict);
  return 0;
}

int snpyio_w_header(const size_t ndim, const size_t *shape, const char dtype[],
                    const bool is_fortran_order, FILE *fp, size_t *header_size) {
  char dict[1024];
  int len = snprintf(dict, sizeof(dict), "{'descr': %s, 'fortran_order': %s, 'shape': (",
                     dtype, is_fortran_order ? "True" : "False");
  for (size_t d = 0; d < ndim; d++) {
    len += snprintf(dict + len, sizeof(dict) - (size_t)len, "%zu,%s", shape[d], (1 == ndim) ? "" : " ");
  }
  len += snprintf(dict + len, sizeof(dict) - (size_t)len, "), }");
  /* pad so that 10 + header_len is a multiple of 64; header ends with '\n' */
  size_t total = 10 + (size_t)len + 1;
  const size_t pad = (64 - total % 64) % 64;
  const size_t hlen = (size_t)len + pad + 1;
  unsigned char pre[10] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0,
                           (unsigned char)(hlen & 0xff), (unsigned char)((hlen >> 8) & 0xff)};
  if (10 != fwrite(pre, 1, 10, fp)) return 1;
  if ((size_t)len != fwrite(dict, 1, (size_t)len, fp)) return 1;
  for (size_t i = 0; i < pad; i++) fputc(' ', fp);
  fputc('\n', fp);
  *header_size = 10 + hlen;
  return 0;
}
