// registry.cpp -- solver plugin registry of the B200 backend.
//
// Same contract as PSuM's src/field_solver/register/registry.cpp:12-21:
// `register_solver` inserts or replaces a table under a name,
// `get_solver_funcs` returns it, or a table with init == NULL for an unknown
// name.  The registry is a function-local static so that backends may
// register from static initialisers in any translation unit.
#include <atomic>
#include <map>
#include <mutex>
#include <string>

#include "common.hpp"

namespace psum_b200 {

namespace {
std::map<std::string, func_table>& registry() {
    static std::map<std::string, func_table> r;
    return r;
}
std::mutex& registry_mutex() {
    static std::mutex m;
    return m;
}
thread_local std::string g_last_error;
std::atomic<unsigned long long> g_launches{0};
thread_local unsigned long long g_thread_launches = 0;
std::once_flag g_mapped_once;
unsigned long long* g_mapped = nullptr;   // pinned host word, device-mapped
}  // namespace

unsigned long long* device_launch_counter() {
    std::call_once(g_mapped_once, [] {
        void* p = nullptr;
        cuda_check(cudaHostAlloc(&p, sizeof(unsigned long long), cudaHostAllocMapped | cudaHostAllocPortable),
                   "cudaHostAlloc launch counter");
        *static_cast<volatile unsigned long long*>(p) = 0ull;
        g_mapped = static_cast<unsigned long long*>(p);
    });
    return g_mapped;
}

void count_launch() {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    ++g_thread_launches;
}
void add_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void uncount_launches(unsigned long long n) { g_launches.fetch_sub(n, std::memory_order_relaxed); }
unsigned long long thread_launches() { return g_thread_launches; }

void set_last_error(const std::string& msg) { g_last_error = msg; }
const std::string& last_error() { return g_last_error; }

}  // namespace psum_b200

extern "C" {

EXPORT void register_solver(const char* name, struct func_table table) {
    if (!name) return;
    std::lock_guard<std::mutex> lk(psum_b200::registry_mutex());
    psum_b200::registry()[name] = table;
}

EXPORT struct func_table get_solver_funcs(const char* name) {
    func_table ans{};
    ans.init = nullptr;
    if (!name) return ans;
    std::lock_guard<std::mutex> lk(psum_b200::registry_mutex());
    auto& reg = psum_b200::registry();
    auto it = reg.find(name);
    if (it != reg.end()) return it->second;
    return ans;
}

EXPORT const char* psum_last_error(void) { return psum_b200::last_error().c_str(); }

EXPORT unsigned long long psum_kernel_launches(void) {
    const volatile unsigned long long* m = psum_b200::g_mapped;
    return psum_b200::g_launches.load() + (m ? *m : 0ull);
}

}
