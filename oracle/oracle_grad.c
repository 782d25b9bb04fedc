/* CPU oracle: adjoint shape gradient. TEST INFRASTRUCTURE ONLY. */
#include <stdint.h>
int oracle_grad_placeholder(void) { return 0; }
