"""vexq_b200: B200 (sm_100a) execution path for vexq's Filter → Project →
HashAggregate / ParallelHashAggregate / ParallelHashJoinAggregate operators.

The product is libvexqcuda.so (C ABI in include/vexq_cuda.h); this package
holds its Python bindings, plan descriptors and seeded data generators."""
