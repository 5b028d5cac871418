// CPU oracle (test infrastructure only): finite-source restatement.
#include "oracle_fs.h"
