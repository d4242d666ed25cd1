"""B200-native XBeach_GPU coupled step (wave action, shallow-water flow,
sediment and bed update) behind the C ABI of include/xbg.h."""
