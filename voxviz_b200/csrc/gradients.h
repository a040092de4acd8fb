// gradients.h - the gradient half of the reference's mip pyramid, densely,
// for small terrains (the lighting path of GigaVoxels.frag).
//
// Leaf level (VolumeDataSet::convert, VoxViz/VoxVizCore/VolumeDataSet.cpp:
// 144-209): the gradient of voxel (x,y,z) is (a(x-1) - a(x+1), a(y-1) -
// a(y+1), a(z-1) - a(z+1)) with a = alpha/255 (binary32) and 0 outside the
// volume, divided by its length (in double, QVector3D arithmetic) when the
// length is positive, else 0; stored as binary32.
// Level m+1 (GenerateMipMap / GetBoxFilterAverage, GigaVoxelsOctTree.cpp:
// 809-960): the 2x2x2 block's gradients summed in binary32 (z, y, x order),
// times 1/8, then QVector3D::normalize (Qt 4.8: in double, left unchanged
// when |len^2 - 1| <= 1e-12 or len^2 <= 1e-12), stored as binary32.
#pragma once

#include <cstdint>
#include <vector>

namespace vv {

class TerrainVolume;

class GradientPyramid {
public:
    // Levels 0 (leaf resolution) .. depth; throws std::length_error above
    // depth 6 (the leaf level alone would be 12 bytes per voxel).
    explicit GradientPyramid(const TerrainVolume& v);
    int dim(int m) const { return dim_[m]; }
    // Gradient of voxel (x,y,z) of level m (zero outside the level).
    void at(int m, int x, int y, int z, float g[3]) const;

private:
    std::vector<std::vector<float>> lv_;
    std::vector<int> dim_;
};

// QVector3D::normalize (Qt 4.8) on binary32 components, in double.
void qt_normalize(float v[3]);

}  // namespace vv
