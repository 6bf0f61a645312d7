"""The fan-out rule of the radix-partitioned group-by (host logic)."""
from bespokeolap_artifacts_b200 import learned as L


def test_fanout_rule():
    assert L.GroupBySizer.fanout(200_000) == 0            # single-pass table (6 MB) stays in L2
    assert L.GroupBySizer.fanout(20_000_000) == 13        # 600 MB table: 8192 partitions of ~2.4K groups
    assert L.GroupBySizer.fanout(0) == 0


def test_join_fanout_rule():
    assert L.JoinSizer.fanout(60_000) == 0            # 1.2 MB single-pass table stays in L2
    assert L.JoinSizer.fanout(30_000_000) == 13       # 600 MB table: 8192 partitions of ~3.7K keys
    assert L.JoinSizer.fanout(-1) == 0
