/* Minimal stand-in for OpenMM's exception type (oracle harness only). */
#ifndef SHIM_OPENMM_EXCEPTION_H_
#define SHIM_OPENMM_EXCEPTION_H_
#include <stdexcept>
#include <string>
namespace OpenMM {
class OpenMMException : public std::runtime_error {
public:
    explicit OpenMMException(const std::string& message) : std::runtime_error(message) {}
};
}
#endif
