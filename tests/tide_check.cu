// Host check of the tide-field header (parahpop_b200/csrc/tide_field.cuh):
// reads known-answer inputs (r[3] v[3] sun[3] moon[3] E[9] mjdUtc ut1Utc
// ttUtc xp yp per line) from stdin and prints, one JSON object per line, the
// solid (zero-tide) and ocean coefficient sets the header forms, in the
// layout of tests/golden/tides_kat.json.
#include <cstdio>
#include <vector>

#include "tide_field.cuh"

using namespace phop::tidefield;

int main() {
    std::vector<OceanAmp> table(kWaves * kSlots);
    buildOceanTable(table.data());
    double v[26];
    for (;;) {
        for (int k = 0; k < 26; ++k)
            if (std::scanf("%lf", &v[k]) != 1) return 0;
        Epoch ep;
        for (int k = 0; k < 3; ++k) {
            ep.sun[k] = v[6 + k];
            ep.moon[k] = v[9 + k];
        }
        for (int k = 0; k < 9; ++k) ep.E[k] = v[12 + k];
        ep.mjdUtc = v[21];
        ep.ut1Utc = v[22];
        ep.ttUtc = v[23];
        ep.xp = v[24];
        ep.yp = v[25];
        double sc[7][7], ss[7][7], oc[7][7], os[7][7];
        tideSetsHost(ep, true, table.data(), sc, ss, oc, os);
        const char* names[4] = {"solidC", "solidS", "oceanC", "oceanS"};
        double(*sets[4])[7] = {sc, ss, oc, os};
        std::printf("{");
        for (int q = 0; q < 4; ++q) {
            std::printf("%s\"%s\":[", q ? "," : "", names[q]);
            for (int n = 0; n < 7; ++n)
                for (int m = 0; m < 7; ++m) std::printf("%s%.17g", (n || m) ? "," : "", sets[q][n][m]);
            std::printf("]");
        }
        std::printf("}\n");
    }
}
