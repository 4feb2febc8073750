// The C++ host side's error behaviour without a device (built and run by tests/test_capi_symbols.py on the CPU):
// bad arguments throw nereus_b200::Error with NB_BAD_INPUT before any device is looked for, and a good call on a
// machine without a device throws NB_NO_DEVICE instead of falling back to the host.
#include <cstdio>
#include <vector>

#include "nereus_b200_solver.hpp"

static int StatusOf(void (*f)())
{
    try
    {
        f();
    }
    catch (const nereus_b200::Error &e)
    {
        return e.status;
    }
    return NB_OK;
}

int main()
{
    int fails = 0;
    auto expect = [&](int got, int want, const char *what) {
        if (got != want)
        {
            std::printf("FAIL %s: status %d, expected %d\n", what, got, want);
            fails++;
        }
    };
    expect(StatusOf([] {
               std::vector<uint8_t> t(27, 2);
               const double o[3] = {0, 0, 0};
               std::vector<double> rows(7 * 4, 0.5);
               nereus_b200::UpdateFluidCells(3, 3, 3, 3, o, 1.0, rows.data() + 1, 4, 0, t.data()); // stride 0
           }),
           NB_BAD_INPUT, "relabel with stride 0");
    expect(StatusOf([] {
               const double o[3] = {0, 0, 0};
               nereus_b200::UpdateFluidCells(3, 3, 3, 3, o, 1.0, nullptr, 0, 7, nullptr); // no labels
           }),
           NB_BAD_INPUT, "relabel without labels");
    expect(StatusOf([] {
               nb_bc_lists L{};
               L.dim = 4; // no such dimension
               nereus_b200::BoundaryReplay bc(0, L);
           }),
           NB_BAD_INPUT, "boundary lists with dim 4");
    expect(StatusOf([] {
               std::vector<uint8_t> t(27, 2);
               const double o[3] = {0, 0, 0};
               std::vector<double> rows(7 * 4, 1.5);
               nereus_b200::UpdateFluidCells(3, 3, 3, 3, o, 1.0, rows.data() + 1, 4, 7, t.data());
           }),
           NB_NO_DEVICE, "relabel without a device");
    std::printf("%s\n", fails ? "FAILED" : "ok");
    return fails ? 1 : 0;
}
