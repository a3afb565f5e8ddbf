/*
 * sma_oracle.c -- instantiates the CPU oracle (sma_oracle_impl.h) in double
 * and in float precision, plus greedy element colouring.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
 * baseline.  Nothing in the product links this file.
 */
#include "sma_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define REAL double
#define SUFFIX _f64
#define SQRT sqrt
#define FABS fabs
#define LOG log
#define POW pow
#define REAL_EPS DBL_EPSILON
#include "sma_oracle_impl.h"
#undef REAL
#undef SUFFIX
#undef SQRT
#undef FABS
#undef LOG
#undef POW
#undef REAL_EPS

#define REAL float
#define SUFFIX _f32
#define SQRT sqrtf
#define FABS fabsf
#define LOG logf
#define POW powf
#define REAL_EPS FLT_EPSILON
#include "sma_oracle_impl.h"

/* First-fit greedy colouring over the element-element graph (elements that
 * share a node are neighbours).  The reference colours the same graph
 * (mod_parall_openmp.f90:557-708 -> graphs_coloring_greedy,
 * mod_graphs.f90:2898-3048) with its own vertex order; any valid colouring
 * gives the same sums per node up to the order of the contributions. */
int orc_color_elements(int nelem, int npoin, const int32_t* lnods,
                       int32_t* color_of, int32_t* color_ptr, int32_t* color_elem)
{
  int32_t* cnt = (int32_t*)calloc((size_t)npoin + 1, sizeof(int32_t));
  for (int64_t k = 0; k < 8 * (int64_t)nelem; ++k) cnt[lnods[k] + 1]++;
  for (int p = 0; p < npoin; ++p) cnt[p + 1] += cnt[p];
  int32_t* adj = (int32_t*)malloc(sizeof(int32_t) * 8 * (size_t)nelem);
  int32_t* pos = (int32_t*)malloc(sizeof(int32_t) * ((size_t)npoin + 1));
  memcpy(pos, cnt, sizeof(int32_t) * ((size_t)npoin + 1));
  for (int e = 0; e < nelem; ++e)
    for (int a = 0; a < 8; ++a) adj[pos[lnods[8 * (int64_t)e + a]]++] = e;
  int ncolor = 0;
  for (int e = 0; e < nelem; ++e) color_of[e] = -1;
  for (int e = 0; e < nelem; ++e) {
    uint64_t used = 0;
    for (int a = 0; a < 8; ++a) {
      int p = lnods[8 * (int64_t)e + a];
      for (int k = cnt[p]; k < cnt[p + 1]; ++k) {
        int c = color_of[adj[k]];
        if (c >= 0 && c < 64) used |= (uint64_t)1 << c;
      }
    }
    int c = 0;
    while (c < 64 && (used >> c) & 1) ++c;
    color_of[e] = c;
    if (c + 1 > ncolor) ncolor = c + 1;
  }
  for (int c = 0; c <= ncolor; ++c) color_ptr[c] = 0;
  for (int e = 0; e < nelem; ++e) color_ptr[color_of[e] + 1]++;
  for (int c = 0; c < ncolor; ++c) color_ptr[c + 1] += color_ptr[c];
  int32_t* fill = (int32_t*)malloc(sizeof(int32_t) * (ncolor > 0 ? ncolor : 1));
  for (int c = 0; c < ncolor; ++c) fill[c] = color_ptr[c];
  for (int e = 0; e < nelem; ++e) color_elem[fill[color_of[e]]++] = e;
  free(fill);
  free(cnt);
  free(adj);
  free(pos);
  return ncolor;
}
