# sed -E script applied to the reference solver (src/main.cpp) when building
# the checker variants in _ref/.  It changes no arithmetic.
#
# 1. Compile-time switches (src/main.cpp:33-38) become overridable with -D.
s/^#define (SUBSTEP_NO|MAX_HORIZON_LENGTH|ABCS_STEP|KINEMATIC_VELOCITY_ABC|THETA_ABC_METHOD) +(-?[0-9]+)(.*)$/#ifndef \1\n#define \1 \2\n#endif/
# 2. VTK writers (src/main.cpp:690,1095-1103) go through macros that
#    -DREF_NO_VTK turns into no-ops; 3. a final-state dump hook.
/^#include "utils.h"/a\
#include <cstdio>\
#ifdef REF_NO_VTK\
#define REF_VTK_vector(...) true\
#define REF_VTK_scalar(...) true\
#else\
#define REF_VTK_vector utils::write_vtk_vector\
#define REF_VTK_scalar utils::write_vtk_scalar\
#endif\
#ifdef REF_DUMP\
#define REF_DUMP_STATE() do { \\\
    FILE *f_ = std::fopen((JobName + Prefix + ".state").c_str(), "wb"); \\\
    if (f_) { int n_ = NodeNo; std::fwrite(&n_, sizeof(int), 1, f_); \\\
      std::fwrite(Un.data(), sizeof(double), 2 * n_, f_); \\\
      std::fwrite(Udn.data(), sizeof(double), 2 * n_, f_); \\\
      std::fwrite(Uddn.data(), sizeof(double), 2 * n_, f_); \\\
      std::fwrite(Theta.data(), sizeof(double), n_, f_); \\\
      std::fwrite(mWeighted.data(), sizeof(double), n_, f_); \\\
      std::fclose(f_); } } while (0)\
#else\
#define REF_DUMP_STATE() do {} while (0)\
#endif
s/utils::write_vtk_(vector|scalar)\(/REF_VTK_\1(/
# The dump runs after the "Time marching took" line, outside the timed loop.
/Time marching took/,/return 0;/ {
  /return 0;/i\
  REF_DUMP_STATE();
}
