"""CPU: the ncu captures that bench.py reports as roofline traffic are present in profiles/ and parse,
for every workload and kernel class it names."""
import bench


def test_traffic_captures_parse():
    for workload, classes in bench.TRAFFIC_CAPTURES.items():
        assert workload in bench.WORKLOADS
        for cls in classes:
            value, scope = bench.captured_traffic(workload, cls)
            assert isinstance(value, int) and value > 0, (workload, cls)
            assert "profiles/" in scope
    assert bench.captured_traffic("interval_box1e5", "no_such_class") == (None, None)
