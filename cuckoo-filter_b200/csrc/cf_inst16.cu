// cf_inst16.cu -- kernel instantiations for 16-bit tags (WordType uint64_t, and uint32_t for the reference's
// word-width comparison geometry).
#include "cf_registry.cuh"

namespace cfb {

void register_bits16(std::vector<OpsTable>& v) {
    v.push_back(Launchers<Cfg<8, 16, 4, 8>>::table());
    v.push_back(Launchers<Cfg<4, 16, 4, 8>>::table());
    v.push_back(Launchers<Cfg<8, 16, 8, 8>>::table());
    v.push_back(Launchers<Cfg<4, 16, 8, 8>>::table());
    v.push_back(Launchers<Cfg<8, 16, 16, 8>>::table());
    v.push_back(Launchers<Cfg<4, 16, 16, 8>>::table());
    v.push_back(Launchers<Cfg<8, 16, 32, 8>>::table());
    v.push_back(Launchers<Cfg<4, 16, 32, 8>>::table());
    v.push_back(Launchers<Cfg<8, 16, 64, 8>>::table());  // 128-byte buckets (cuckoo_bucket_size.cu:78)
    v.push_back(Launchers<Cfg<4, 16, 64, 8>>::table());
    v.push_back(Launchers<Cfg<8, 16, 128, 8>>::table());  // 256-byte buckets
    v.push_back(Launchers<Cfg<4, 16, 128, 8>>::table());
    v.push_back(Launchers<Cfg<8, 16, 16, 4>>::table());  // WordType uint32_t
    v.push_back(Launchers<Cfg<4, 16, 16, 4>>::table());  // WordType uint32_t
    // AddSub and Offset alternate-bucket policies (bucket_policy_benchmark.cu:16-17)
    v.push_back(Launchers<Cfg<8, 16, 16, 8, ALT_ADDSUB>>::table());
    v.push_back(Launchers<Cfg<4, 16, 16, 8, ALT_ADDSUB>>::table());
    v.push_back(Launchers<Cfg<8, 16, 16, 8, ALT_OFFSET>>::table());
    v.push_back(Launchers<Cfg<4, 16, 16, 8, ALT_OFFSET>>::table());
}

}  // namespace cfb
