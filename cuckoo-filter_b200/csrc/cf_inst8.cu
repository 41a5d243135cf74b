// cf_inst8.cu -- kernel instantiations for 8-bit tags (WordType uint64_t, and uint32_t for the reference's
// word-width comparison geometry).
#include "cf_registry.cuh"

namespace cfb {

void register_bits8(std::vector<OpsTable>& v) {
    v.push_back(Launchers<Cfg<8, 8, 8, 8>>::table());
    v.push_back(Launchers<Cfg<4, 8, 8, 8>>::table());
    v.push_back(Launchers<Cfg<8, 8, 16, 8>>::table());
    v.push_back(Launchers<Cfg<4, 8, 16, 8>>::table());
    v.push_back(Launchers<Cfg<8, 8, 32, 8>>::table());
    v.push_back(Launchers<Cfg<4, 8, 32, 8>>::table());
    v.push_back(Launchers<Cfg<8, 8, 64, 8>>::table());
    v.push_back(Launchers<Cfg<4, 8, 64, 8>>::table());
    v.push_back(Launchers<Cfg<8, 8, 16, 4>>::table());  // WordType uint32_t
    v.push_back(Launchers<Cfg<4, 8, 16, 4>>::table());  // WordType uint32_t
}

}  // namespace cfb
