// CPU oracle (test infrastructure only): finite-source restatement.  Filled in below.
#pragma once
