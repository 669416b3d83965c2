/* oracle_util.c - thread control of the CPU oracle (test infrastructure). */
#include <omp.h>

void oracle_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int oracle_max_threads(void) { return omp_get_max_threads(); }
