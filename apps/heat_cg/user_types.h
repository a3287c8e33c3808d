/* Types and helpers shared by the host code and the kernels of the CG heat
 * conduction driver (OPS convention: user_types.h). */
#ifndef HEAT_CG_USER_TYPES_H
#define HEAT_CG_USER_TYPES_H

#ifndef OPS_FUN_PREFIX
#define OPS_FUN_PREFIX
#endif

/* U[0,1) from a counter-based hash (splitmix64 finaliser) of the seed and a
 * 2D index: the same bits on the host and on the device. */
static inline OPS_FUN_PREFIX double hc_uniform(int seed, int i, int j) {
  unsigned long long z = ((unsigned long long)(unsigned)seed << 42) ^
                         ((unsigned long long)(unsigned)i << 21) ^ (unsigned long long)(unsigned)j;
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

#endif
