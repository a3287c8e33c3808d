/* Helpers shared by the host code and kernels of the opsunit application. */
#ifndef OPSUNIT_USER_TYPES_H
#define OPSUNIT_USER_TYPES_H

#ifndef OPS_FUN_PREFIX
#define OPS_FUN_PREFIX
#endif

/* small deterministic perturbation in [0, 1/1024) so fields are not affine */
static inline OPS_FUN_PREFIX double ou_hash(int i, int j) {
  unsigned int h = (unsigned int)(i * 73856093) ^ (unsigned int)(j * 19349663);
  h ^= h >> 13;
  h *= 0x5bd1e995u;
  h ^= h >> 15;
  return (double)(h & 1023u) / 1048576.0;
}

#endif
