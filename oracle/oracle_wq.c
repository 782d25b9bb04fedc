/* CPU oracle: weighted-quadrature path (filled in below). TEST INFRASTRUCTURE ONLY. */
#include <stdint.h>
int oracle_wq_placeholder(void) { return 0; }
