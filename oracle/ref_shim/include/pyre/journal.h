// Minimal stand-in for pyre's journal (test infrastructure: it lets the reference's CPU correlator
// compile unmodified).  The reference writes progress and per-pair timings to named channels
// (info_t, debug_t) with `channel << pyre::journal::at(__HERE__) << ... << pyre::journal::endl`.
// Here every channel accepts and discards what it is given; the operands are still evaluated,
// as they are in pyre.
#ifndef AMPCOR_REF_SHIM_PYRE_JOURNAL_H
#define AMPCOR_REF_SHIM_PYRE_JOURNAL_H

#ifndef __HERE__
#define __HERE__ __FILE__, __LINE__, __func__
#endif

namespace pyre {
namespace journal {

struct location_t {};
inline location_t at(const char*, int, const char*) { return {}; }

struct newline_t {};
struct endl_t {};
inline constexpr newline_t newline{};
inline constexpr endl_t endl{};

class channel_t {
public:
    explicit channel_t(const char*) {}
    template <typename T>
    channel_t& operator<<(const T&) { return *this; }
};

using debug_t = channel_t;
using info_t = channel_t;
using warning_t = channel_t;
using error_t = channel_t;
using firewall_t = channel_t;

}  // namespace journal
}  // namespace pyre

#endif
