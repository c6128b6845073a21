/* les_oracle.c -- TEST INFRASTRUCTURE: LES (AMD, les_model_type 5)
 * restatement; filled in with the LES path. */
#include "oracle.h"
