// Registry of the GPU contexts attached to the reference's SlaterDet objects.
#include "qbx_shim.h"

#include <cstdlib>
#include <map>
#include <mutex>
#include <string>

#include "SlaterDet.h"

namespace qbx_shim {

namespace {
std::mutex g_mu;
std::map<const SlaterDet*, qbx_context*>& registry() {
  static std::map<const SlaterDet*, qbx_context*> r;
  return r;
}
}  // namespace

void attach(const SlaterDet& sd, qbx_context* q) {
  std::lock_guard<std::mutex> lock(g_mu);
  registry()[&sd] = q;
}

void detach(const SlaterDet& sd) {
  std::lock_guard<std::mutex> lock(g_mu);
  registry().erase(&sd);
}

qbx_context* context_of(const SlaterDet& sd) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = registry().find(&sd);
  if (it == registry().end())
    throw SlaterDetException("no GPU context attached to this SlaterDet (qbx_shim::attach)");
  return it->second;
}

void check(qbx_context* q, int rc) {
  if (rc) throw SlaterDetException(std::string("qbx: ") + qbx_last_error(q));
}

int device() {
  const char* e = std::getenv("QBX_DEVICE");
  return e ? std::atoi(e) : 0;
}

}  // namespace qbx_shim
