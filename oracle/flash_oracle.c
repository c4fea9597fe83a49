/* TEST INFRASTRUCTURE ONLY (see oracle.h). Pure-component PR HEM UV flash restatement. */
#include "oracle.h"
