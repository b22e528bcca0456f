/* Minimal stand-in for OpenMM's osrngseed() (oracle harness only): a fixed nonzero seed. */
#ifndef SHIM_OPENMM_OSRNGSEED_H_
#define SHIM_OPENMM_OSRNGSEED_H_
namespace OpenMM {
inline int osrngseed() { return 20260101; }
}
#endif
