/* Minimal stand-in for MATLAB's mex.h, enough to compile the reference's
 * host-side Goldstein linker sources outside MATLAB (test infrastructure).
 * Only the message functions they reference are provided, as no-ops. */
#ifndef ORACLE_STUB_MEX_H
#define ORACLE_STUB_MEX_H
inline int mexPrintf(const char*, ...) { return 0; }
inline int mexEvalString(const char*) { return 0; }
#endif
