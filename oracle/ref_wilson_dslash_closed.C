// Test infrastructure only.  The reference's serial wilson_dslash.C ends the
// body of wilson_dslash() without its closing brace (the namespace-closing
// macro at its line 518 closes the function instead).  This translation unit
// compiles that file unchanged and supplies the missing brace afterwards,
// which closes the namespace the file left open.
#include "src/util/dirac_op/d_op_wilson/noarch/wilson_dslash.C"
}
