// No-op timer stand-in for the absent phiprof library (oracle builds only).
#pragma once
#include <string>
namespace phiprof {
inline int initializeTimer(const std::string&, ...) { return 0; }
struct Timer {
   template <typename... A> explicit Timer(A&&...) {}
   void stop() {}
};
}  // namespace phiprof
