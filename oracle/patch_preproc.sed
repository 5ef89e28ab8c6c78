# sed -E script applied to the reference preprocessor (preprocessor/main.cpp)
# when building checker variants in _ref/.  It only makes the hard-coded
# domain radius, grid spacing and m-ratio (preprocessor/main.cpp:64-67)
# overridable with -DREF_DOMAIN_RADIUS=, -DREF_DX=, -DREF_M=.  Arithmetic is
# unchanged.
s/^static const double DOMAIN_RADIUS = ([0-9.]+);(.*)$/#ifndef REF_DOMAIN_RADIUS\n#define REF_DOMAIN_RADIUS \1\n#endif\nstatic const double DOMAIN_RADIUS = REF_DOMAIN_RADIUS;\2/
s/^static const double DX = ([0-9.]+);(.*)$/#ifndef REF_DX\n#define REF_DX \1\n#endif\nstatic const double DX = REF_DX;\2/
s/^static const double DY = ([0-9.]+);(.*)$/static const double DY = REF_DX;\2/
s/^static const double DELTA = ([0-9.]+) \* DX;(.*)$/#ifndef REF_M\n#define REF_M \1\n#endif\nstatic const double DELTA = REF_M * DX;\2/
