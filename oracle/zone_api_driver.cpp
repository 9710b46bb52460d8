// Test driver of the per-zone API of the reference's include/zone_pass.h (build_zone_layout,
// build_particle_ids_in_zone, run_zone_kernel_inplace). Test infrastructure: oracle/Makefile
// compiles it twice, against the reference's own sources (_ref/zone_api_ref) and against the
// C++ shim over libmpcd_b200.so (_ref/zone_api_b200); tests/test_zone_api.py runs both on
// the same case and compares every file they write. It uses only the reference's headers.
//
//   zone_api_* params.kv in_x.bin in_v.bin out_prefix mode seed_base stride
//
// Writes <out_prefix>layout.bin (zone count, then per zone: id, cell count, cell ids; then the
// owner map) and, for every stride-th zone z: <out_prefix>zone<z>_ids.bin (its particle ids),
// _x.bin / _v.bin (the state after run_zone_kernel_inplace on a copy of the input, with seed
// seed_base + 104729 (z + 1)) and _stats.bin (stats[6], diag[10], movedDense, movedSparse as
// doubles).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "params_io.h"
#include "state_io.h"
#include "types.h"
#include "zone_pass.h"

namespace {

template <typename T>
void put(std::ofstream& f, const T& v) {
    f.write(reinterpret_cast<const char*>(&v), sizeof v);
}

template <typename T>
void put_all(const std::string& path, const std::vector<T>& a) {
    std::ofstream f(path, std::ios::binary);
    if (!a.empty()) f.write(reinterpret_cast<const char*>(a.data()), (std::streamsize)(a.size() * sizeof(T)));
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 8) {
        std::cerr << "usage: zone_api params.kv in_x.bin in_v.bin out_prefix mode seed_base stride\n";
        return 2;
    }
    try {
        const mpcd::Params params = mpcd::read_params_kv(argv[1]);
        const mpcd::State s = mpcd::read_state(argv[2], argv[3], "", "", false, false, params.n);
        const std::string out = argv[4];
        const std::string mode = argv[5];
        const std::uint64_t seedBase = std::strtoull(argv[6], nullptr, 10);
        const int stride = std::atoi(argv[7]);

        const mpcd::ZoneLayout L = mpcd::build_zone_layout(params, mode);
        {
            std::ofstream f(out + "layout.bin", std::ios::binary);
            put(f, (std::int32_t)L.zones.size());
            for (const auto& z : L.zones) {
                put(f, (std::int32_t)z.id);
                put(f, (std::int32_t)z.cellIds.size());
                for (int c : z.cellIds) put(f, (std::int32_t)c);
                std::int32_t nm = 0;
                for (char m : z.maskVec) nm += m ? 1 : 0;
                put(f, nm);
            }
            for (std::int32_t o : L.ownerMap) put(f, o);
        }
        for (std::size_t z = 0; z < L.zones.size(); z += (std::size_t)(stride > 0 ? stride : 1)) {
            const auto& zone = L.zones[z];
            const std::string pre = out + "zone" + std::to_string(z);
            put_all(pre + "_ids.bin", mpcd::build_particle_ids_in_zone(s.x, params, zone));
            std::vector<double> x = s.x, v = s.v;
            const mpcd::ZoneKernelStats st =
                mpcd::run_zone_kernel_inplace(x, v, params, zone, seedBase + 104729ULL * (std::uint64_t)(z + 1));
            put_all(pre + "_x.bin", x);
            put_all(pre + "_v.bin", v);
            std::vector<double> sd(st.stats.begin(), st.stats.end());
            sd.insert(sd.end(), st.diag.begin(), st.diag.end());
            sd.push_back((double)st.movedDense);
            sd.push_back((double)st.movedSparse);
            put_all(pre + "_stats.bin", sd);
        }
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
