/*
 * Dat dump through the public OPS API, for parity checks between backends.
 *
 * dump_dats() fetches each dat's interior with ops_dat_get_extents and
 * ops_dat_fetch_data (the data-access calls of ops_lib_core.h, implemented
 * by the reference in core/ops_dummy_singlenode.cpp:737-765 and by this
 * backend in its runtime), so the same call works unchanged on this
 * backend, on the CPU oracle and on the reference's own sequential and
 * OpenMP backends.
 *
 * Record format (the one tests/opsdump.py reads): "DAT0", name length +
 * name, type length + type, dim, type size, ndims, soa flag, size[5],
 * d_m[5], d_p[5], byte count, data.  The sizes written are the interior
 * extents and d_m = d_p = 0, since ops_dat_fetch_data returns the interior
 * without halos (x fastest, components interleaved).
 */
#ifndef APPS_DUMPDATS_H
#define APPS_DUMPDATS_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static inline int dump_dats(const char *path, ops_dat *dats, int n) {
  FILE *f = fopen(path, "wb");
  if (!f) return -1;
  for (int i = 0; i < n; i++) {
    ops_dat d = dats[i];
    if (!d) continue;
    const int nd = d->block->dims;
    int disp[5] = {0, 0, 0, 0, 0}, ext[5] = {1, 1, 1, 1, 1};
    ops_dat_get_extents(d, 0, disp, ext);
    size_t pts = 1;
    for (int k = 0; k < nd; k++) pts *= (size_t)ext[k];
    const int ts = d->elem_size / d->dim;
    const size_t nbytes = pts * (size_t)d->elem_size;
    char *buf = (char *)malloc(nbytes ? nbytes : 1);
    if (!buf) {
      fclose(f);
      return -2;
    }
    ops_dat_fetch_data(d, 0, buf);
    const int nl = (int)strlen(d->name), tl = (int)strlen(d->type);
    int hdr[4] = {d->dim, ts, nd, 0};
    int size[5] = {1, 1, 1, 1, 1}, zero[5] = {0, 0, 0, 0, 0};
    for (int k = 0; k < nd; k++) size[k] = ext[k];
    unsigned long long nb = nbytes;
    fwrite("DAT0", 1, 4, f);
    fwrite(&nl, sizeof(int), 1, f);
    fwrite(d->name, 1, nl, f);
    fwrite(&tl, sizeof(int), 1, f);
    fwrite(d->type, 1, tl, f);
    fwrite(hdr, sizeof(int), 4, f);
    fwrite(size, sizeof(int), 5, f);
    fwrite(zero, sizeof(int), 5, f);
    fwrite(zero, sizeof(int), 5, f);
    fwrite(&nb, sizeof(nb), 1, f);
    fwrite(buf, 1, nbytes, f);
    free(buf);
  }
  return fclose(f) == 0 ? 0 : -3;
}

#endif /* APPS_DUMPDATS_H */
