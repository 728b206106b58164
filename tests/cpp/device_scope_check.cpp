// Checks bph::DeviceScopeT (bipoly_hydro_b200/csrc/bph_device_scope.h)
// against a fake runtime that records the current device: the caller's
// device comes back at scope exit, no switch happens when the context's
// device is already current, and a failed switch restores nothing.
#include <cstdio>
#include <vector>

#include "bph_device_scope.h"

namespace {
struct FakeRt {
    using err_t = int;
    static constexpr int ok = 0;
    static int current;
    static int fail_set_to;  // set() to this ordinal fails
    static std::vector<int> sets;
    static int get(int *d) {
        *d = current;
        return ok;
    }
    static int set(int d) {
        sets.push_back(d);
        if (d == fail_set_to) return 101;
        current = d;
        return ok;
    }
};
int FakeRt::current = 0;
int FakeRt::fail_set_to = -1;
std::vector<int> FakeRt::sets;

int failures = 0;
void expect(bool ok, const char *what) {
    if (!ok) {
        std::printf("FAIL: %s\n", what);
        ++failures;
    }
}
}  // namespace

int main() {
    using Scope = bph::DeviceScopeT<FakeRt>;
    // switch to device 3 from 1, restore 1
    FakeRt::current = 1;
    {
        Scope s(3);
        expect(s.status() == 0, "status ok");
        expect(s.previous() == 1, "previous ordinal saved");
        expect(FakeRt::current == 3, "context device current inside the scope");
    }
    expect(FakeRt::current == 1, "caller's device restored");
    expect(FakeRt::sets.size() == 2 && FakeRt::sets[0] == 3 && FakeRt::sets[1] == 1, "one switch and one restore");
    // same device: no set() at all
    FakeRt::sets.clear();
    FakeRt::current = 2;
    {
        Scope s(2);
        expect(s.status() == 0, "status ok (same device)");
    }
    expect(FakeRt::sets.empty(), "no switch when the device is already current");
    expect(FakeRt::current == 2, "device unchanged");
    // nested scopes unwind in order
    FakeRt::current = 0;
    {
        Scope a(1);
        {
            Scope b(2);
            expect(FakeRt::current == 2, "inner scope device");
        }
        expect(FakeRt::current == 1, "outer scope device after inner exit");
    }
    expect(FakeRt::current == 0, "outermost caller device restored");
    // failed switch: status reports it, nothing restored
    FakeRt::sets.clear();
    FakeRt::current = 0;
    FakeRt::fail_set_to = 5;
    {
        Scope s(5);
        expect(s.status() == 101, "failed switch reported");
    }
    expect(FakeRt::current == 0, "device untouched after a failed switch");
    expect(FakeRt::sets.size() == 1, "no restore call after a failed switch");
    if (failures == 0) std::printf("device scope: all checks passed\n");
    return failures == 0 ? 0 : 1;
}
