// Drop-in check of the C++ front end: the calling pattern of the reference's
// own tester (tests/src/main.cpp:1526-1621 of hakarlss/Voxelizer) compiled
// against include/vox/voxelizer.h and libvxb.so.  Reads a mesh from a raw
// file (uint32 nV, nT; float vertices[3nV]; uint32 indices[3nT];
// uint8 materials[nT]), runs voxelizeToNodesToRAM / voxelizeToRAM / the
// device-pointer voxelizeToNodes, a slice, devConfig partitions and
// simulateMultidevice, and writes the results for the Python test to compare
// with the C ABI.
#include <vox/voxelizer.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s mesh.bin out_prefix\n", argv[0]);
        return 2;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    uint32_t nV = 0, nT = 0;
    if (std::fread(&nV, 4, 1, f) != 1 || std::fread(&nT, 4, 1, f) != 1) return 4;
    std::vector<float> v(3 * (size_t)nV);
    std::vector<vox::uint> idx(3 * (size_t)nT);
    std::vector<vox::uchar> mats(nT);
    if (std::fread(v.data(), 4, v.size(), f) != v.size()) return 5;
    if (std::fread(idx.data(), 4, idx.size(), f) != idx.size()) return 6;
    if (std::fread(mats.data(), 1, mats.size(), f) != mats.size()) return 7;
    std::fclose(f);

    std::string pre(argv[2]);
    try {
        vox::Voxelizer<vox::LongNode> voxelizer(v.data(), idx.data(), nV, nT);
        voxelizer.setMaterials(mats.data(), 8);
        voxelizer.setMaterialOutput(true);
        vox::NodePointer<vox::LongNode> res = voxelizer.voxelizeToNodesToRAM(80u);
        size_t n = (size_t)res.dim.x * res.dim.y * res.dim.z;
        FILE* o = std::fopen((pre + "_nodes.bin").c_str(), "wb");
        std::fwrite(&res.dim, sizeof(res.dim), 1, o);
        std::fwrite(res.ptr, sizeof(vox::LongNode), n, o);
        std::fclose(o);
        delete[] res.ptr;

        // Device pointers, released to the caller (cudaFree), as the reference.
        std::vector<vox::NodePointer<vox::LongNode> > dres = voxelizer.voxelizeToNodes(80u);
        std::vector<vox::LongNode> back(n);
        cudaMemcpy(back.data(), dres[0].ptr, n * sizeof(vox::LongNode), cudaMemcpyDeviceToHost);
        cudaFree(dres[0].ptr);
        o = std::fopen((pre + "_nodes_dev.bin").c_str(), "wb");
        std::fwrite(back.data(), sizeof(vox::LongNode), n, o);
        std::fclose(o);

        // A slice along y (voxelizeSliceToRAM) and devConfig partitions, as
        // device pointers and, inside simulateMultidevice, host arrays.
        vox::NodePointer<vox::LongNode> sl = voxelizer.voxelizeSliceToRAM(80u, 1, 20);
        size_t ns = (size_t)sl.dim.x * sl.dim.y * sl.dim.z;
        o = std::fopen((pre + "_slice.bin").c_str(), "wb");
        std::fwrite(&sl.dim, sizeof(sl.dim), 1, o);
        std::fwrite(sl.ptr, sizeof(vox::LongNode), ns, o);
        std::fclose(o);
        delete[] sl.ptr;
        std::vector<vox::NodePointer<vox::LongNode> > parts = voxelizer.voxelizeToNodes(80u, make_uint2(2, 2));
        o = std::fopen((pre + "_parts.bin").c_str(), "wb");
        for (auto& pp : parts) {
            size_t np = (size_t)pp.dim.x * pp.dim.y * pp.dim.z;
            std::vector<vox::LongNode> hb(np);
            cudaMemcpy(hb.data(), pp.ptr, np * sizeof(vox::LongNode), cudaMemcpyDeviceToHost);
            cudaFree(pp.ptr);
            std::fwrite(&pp.dim, sizeof(pp.dim), 1, o);
            std::fwrite(&pp.loc, sizeof(pp.loc), 1, o);
            std::fwrite(hb.data(), sizeof(vox::LongNode), np, o);
        }
        std::fclose(o);
        std::vector<vox::NodePointer<vox::LongNode> > sim = voxelizer.simulateMultidevice(
            [&]() { return voxelizer.voxelizeToNodes(80u, make_uint2(2, 1)); });
        o = std::fopen((pre + "_sim.bin").c_str(), "wb");
        for (auto& pp : sim) {
            size_t np = (size_t)pp.dim.x * pp.dim.y * pp.dim.z;
            std::fwrite(&pp.dim, sizeof(pp.dim), 1, o);
            std::fwrite(&pp.loc, sizeof(pp.loc), 1, o);
            std::fwrite(pp.ptr, sizeof(vox::LongNode), np, o);   // host arrays inside simulateMultidevice
            delete[] pp.ptr;
        }
        std::fclose(o);

        // Plain bit array through a fresh instance (node output off).
        vox::Voxelizer<vox::ShortNode> plain(v.data(), idx.data(), nV, nT);
        vox::NodePointer<vox::ShortNode> bits = plain.voxelizeToRAM(80u);
        size_t words = (size_t)bits.dim.x * bits.dim.y * bits.dim.z / 32;
        o = std::fopen((pre + "_bits.bin").c_str(), "wb");
        std::fwrite(&bits.dim, sizeof(bits.dim), 1, o);
        std::fwrite(bits.vptr, 4, words, o);
        std::fclose(o);
        delete[] bits.vptr;

        // Errors surface as vox::Exception, as in the reference.
        bool threw = false;
        try {
            vox::Voxelizer<vox::ShortNode> bad(v.data(), idx.data(), nV, nT);
            bad.setMaterials(mats.data(), 9);
        } catch (const vox::Exception& e) {
            threw = true;
        }
        if (!threw) return 8;
        // FCC nodes refuse maxDimension sizing with a message and an empty result.
        vox::Voxelizer<vox::ShortFCCNode> fcc(v.data(), idx.data(), nV, nT);
        vox::NodePointer<vox::ShortFCCNode> none = fcc.voxelizeToNodesToRAM(80u);
        if (none.ptr != nullptr) return 9;
    } catch (const vox::Exception& e) {
        std::fprintf(stderr, "vox::Exception: %s\n", e.what());
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
