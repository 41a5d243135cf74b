// cf_inst32.cu -- kernel instantiations for 32-bit tags (WordType uint64_t, and uint32_t for the reference's
// word-width comparison geometry).
#include "cf_registry.cuh"

namespace cfb {

void register_bits32(std::vector<OpsTable>& v) {
    v.push_back(Launchers<Cfg<8, 32, 2, 8>>::table());
    v.push_back(Launchers<Cfg<4, 32, 2, 8>>::table());
    v.push_back(Launchers<Cfg<8, 32, 4, 8>>::table());
    v.push_back(Launchers<Cfg<4, 32, 4, 8>>::table());
    v.push_back(Launchers<Cfg<8, 32, 8, 8>>::table());
    v.push_back(Launchers<Cfg<4, 32, 8, 8>>::table());
    v.push_back(Launchers<Cfg<8, 32, 16, 8>>::table());
    v.push_back(Launchers<Cfg<4, 32, 16, 8>>::table());
    v.push_back(Launchers<Cfg<8, 32, 8, 4>>::table());  // WordType uint32_t
    v.push_back(Launchers<Cfg<4, 32, 8, 4>>::table());  // WordType uint32_t
}

}  // namespace cfb
