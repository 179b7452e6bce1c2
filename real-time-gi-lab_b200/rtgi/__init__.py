"""rtgi: host side of the B200 GI hot path (voxel clipmap rebuild, voxel DDA radiance cascades, merge and gather).

Mirrors the reference renderer's host objects for that path (src/core/voxel.ts VoxWorld, src/core/rc.ts Rc,
src/core/frame.ts packFrame, src/runner/configs.ts parseConfig) over the C-ABI library libgi_b200.so.
"""
