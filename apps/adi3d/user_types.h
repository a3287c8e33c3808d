/* Helpers shared by host code and kernels of the 3D ADI driver. */
#ifndef ADI3D_USER_TYPES_H
#define ADI3D_USER_TYPES_H

#ifndef OPS_FUN_PREFIX
#define OPS_FUN_PREFIX
#endif

/* U[0,1) from a counter-based hash (splitmix64 finaliser) of the seed and
 * the 3D global index: identical bits on the host and on the device. */
static inline OPS_FUN_PREFIX double adi_uniform(int seed, const int *idx) {
  unsigned long long z = ((unsigned long long)(unsigned)seed << 48) ^
                         ((unsigned long long)(unsigned)idx[2] << 32) ^
                         ((unsigned long long)(unsigned)idx[1] << 16) ^
                         (unsigned long long)(unsigned)idx[0];
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

#endif
