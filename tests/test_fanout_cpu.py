"""The fan-out rule of the radix-partitioned group-by (host logic)."""
from bespokeolap_artifacts_b200 import learned as L


def test_fanout_rule():
    assert L.GroupBySizer.fanout(200_000) == 0            # single-pass table (6 MB) stays in L2
    assert L.GroupBySizer.fanout(20_000_000) == 13        # 600 MB table: 8192 partitions of ~2.4K groups
    assert L.GroupBySizer.fanout(0) == 0
