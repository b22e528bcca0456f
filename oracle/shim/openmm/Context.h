/* Minimal stand-in for OpenMM's Context declaration (oracle harness only). */
#ifndef SHIM_OPENMM_CONTEXT_H_
#define SHIM_OPENMM_CONTEXT_H_
namespace OpenMM {
class Context;
}
#endif
