// lattice_fname.h -- forced include for the reference's src/alg/lattice.C in
// its GPU configuration only.  Under USE_GPU, Lattice::Mean and
// Lattice::Variance pass an undeclared `fname` to ERR.NotImplemented
// (lattice.C:167,187), so the file does not compile as shipped.  It is built
// with -Dfname=nrcps_fname: the functions that declare their own name keep
// it (the local shadows this global), the two that do not get this one.
extern const char* nrcps_fname;
