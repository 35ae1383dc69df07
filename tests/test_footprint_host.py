"""Host-only admission arithmetic of the serving layer: the footprint of a batch grows by exactly
the deterministic mode's accumulators (64 B per degree of freedom, 24 B per instance) when that
mode is on. No GPU is needed: the library's footprint functions are host arithmetic."""
import pytest


@pytest.mark.parametrize("model,sizes,dofs", [("voronoi", [100, 4096, 333], 100 + 4096 + 333),
                                              ("vertex", [100, 2000], 2 * (100 + 2000))])
def test_deterministic_footprint(cglib, model, sizes, dofs):
    from cellgpu_b200.serve import footprint
    base = footprint(model, sizes)
    det = footprint(model, sizes, deterministic=True)
    assert det - base == 64 * dofs + 24 * len(sizes)
    assert footprint(model, sizes + [50]) > base
